// The C ABI of libkascade_b200.so (declared in include/kascade_b200.h).
#include <cstddef>
#include <cstring>
#include <new>

#include "gen_common.h"
#include "ranker.cuh"

namespace ks {
kascade_status root_forest_impl(kascade_ctx& ctx, const uint64_t* parent, uint32_t n, uint64_t* root_out,
                                uint64_t* depth_out, int keep_roots, const Params& p, cudaStream_t s, bool device_levels = false);
kascade_status compute_euler_tour_impl(kascade_ctx& ctx, const uint64_t* parent, uint32_t n, uint64_t* tour,
                                       uint64_t* m_out, cudaStream_t s);
kascade_status gen_list(uint64_t n, uint64_t seed, uint32_t layout, uint64_t* succ, cudaStream_t s);
kascade_status gen_weights(uint64_t n, uint64_t seed, uint32_t wbits, uint32_t* w, cudaStream_t s);
kascade_status gen_forest(uint64_t n, uint64_t seed, uint32_t kind, uint64_t blocks, uint64_t spine, uint64_t* parent,
                          cudaStream_t s);
kascade_status initial_state(kascade_ctx& ctx, const uint64_t* succ, uint64_t n, uint64_t* root, int64_t* rank,
                             cudaStream_t s);
kascade_status pack_impl(kascade_ctx& ctx, const uint64_t* succ, const int64_t* rank, uint64_t n,
                         const uint64_t* active, uint64_t k, uint64_t* succ_packed, int64_t* rank_packed,
                         cudaStream_t s);
kascade_status unpack_impl(kascade_ctx& ctx, const uint64_t* succ_packed, const int64_t* rank_packed,
                           const uint64_t* active, uint64_t k, uint64_t* succ, int64_t* rank, uint64_t n,
                           cudaStream_t s);
kascade_status rank_batch_impl(kascade_ctx& ctx, const kascade_segment* segs, uint32_t nseg, const uint64_t* in,
                               const uint32_t* weights, uint64_t total, uint64_t* root_out, uint64_t* rank_out,
                               const kascade_opts* opts, cudaStream_t s, bool device_levels);
}  // namespace ks

using namespace ks;

namespace {

constexpr uint64_t MAX_LIST = 0xFFFFFFFEull;
constexpr uint64_t MAX_FOREST = 0x7FFFFFFFull;

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

kascade_status begin_call(kascade_ctx* ctx, cudaStream_t s, const kascade_opts* o) {
  if (!ctx) return KASCADE_ERR_INVALID_ARG;
  // callers built against the first version of kascade_opts (without
  // level0_mode / max_chain) pass a smaller struct_size; both are accepted
  if (o && o->struct_size != 0 && o->struct_size < offsetof(kascade_opts, level0_mode)) return KASCADE_ERR_INVALID_ARG;
  KS_CUDA(ensure_device(ctx->device));
  if (ctx->done_event && ctx->last_stream != s) KS_CUDA(cudaStreamWaitEvent(s, ctx->done_event, 0));
  KS_TRY(arena_begin_call(*ctx, s));
  KS_TRY(status_reset(*ctx, s));
  ctx->profile = o && o->profile;
  ctx->async_pending = false;
  ctx->host_rerun.set = false;
  ctx->pending_levels = 0;
  return KASCADE_OK;
}

kascade_status end_call(kascade_ctx* ctx, cudaStream_t s, kascade_status st, const kascade_opts* o) {
  cudaEventRecord(ctx->done_event, s);
  ctx->last_stream = s;
  if (st != KASCADE_OK) {
    // a host-side error: let the enqueued work drain before reporting
    cudaStreamSynchronize(s);
    cudaGetLastError();
    ctx->last_status = st;
    return st;
  }
  if (o && o->async) {
    ctx->async_pending = true;
    return KASCADE_OK;
  }
  return status_finish(*ctx, s);
}

// device_levels: the ruling-set recursion keeps its level sizes on the device
// (no host wait inside the call); a list it cannot hold reports
// KASCADE_ERR_TIMEOUT and the caller reruns without it.  Only for calls whose
// outputs are not their inputs (the rerun needs the inputs intact).
kascade_status rank_list_generic(kascade_ctx& ctx, const uint64_t* succ, WKind wk, const void* w, uint64_t n,
                                 uint64_t* root_out, uint64_t* rank_out, int keep_roots, const Params& p,
                                 cudaStream_t s, bool device_levels = false) {
  if (n == 0) return KASCADE_OK;
  if (n > MAX_LIST) return KASCADE_ERR_TOO_LARGE;
  Rec* rec = alloc<Rec>(ctx, n);
  uint32_t* ruler_elem = alloc<uint32_t>(ctx, n);
  if (!rec || !ruler_elem) return KASCADE_ERR_OOM;
  if (device_levels && p.algorithm == KASCADE_ALGO_SPARSE_RULING_SET && n > p.base_max && p.max_levels > 0) {
    uint32_t* r_dev = nullptr;
    SinkPlain sink{root_out, rank_out, keep_roots};
    if (n < p.level0_log_min) {
      KS_TRY(prepare_arrays(ctx, succ, wk, w, (uint32_t)n, rec, ruler_elem, nullptr, p, s, &r_dev));
      return rank_records_dev(ctx, rec, (uint32_t)n, r_dev, dev_cap_next((uint32_t)n, p.spacing0), ruler_elem,
                              sink, p, s);
    }
    if (!keep_roots) {
      // the write-free level 0 with the ruler count and the deeper levels on the device
      KS_TRY(prepare_arrays(ctx, succ, wk, w, (uint32_t)n, rec, ruler_elem, nullptr, p, s, &r_dev));
      return rank_level0_log(ctx, rec, (uint32_t)n, dev_cap_next((uint32_t)n, p.spacing0), ruler_elem,
                             sink.log_target((uint32_t)n), p, s, r_dev);
    }
  }
  uint32_t r0 = 0;
  KS_TRY(prepare_arrays(ctx, succ, wk, w, (uint32_t)n, rec, ruler_elem, &r0, p, s));
  SinkPlain sink{root_out, rank_out, keep_roots};
  if (p.algorithm == KASCADE_ALGO_SPARSE_RULING_SET)
    return rank_records(ctx, rec, (uint32_t)n, r0, ruler_elem, sink, p, s);
  ctx.last_levels.clear();
  ctx.last_levels.push_back(n);
  return pointer_double_records(ctx, rec, (uint32_t)n, nullptr, sink, s);
}

kascade_status validate_list(kascade_ctx& ctx, const uint64_t* succ, uint64_t n, const kascade_opts* o,
                              const Params& p, cudaStream_t s) {
  if (!o || !o->validate || p.algorithm != KASCADE_ALGO_SPARSE_RULING_SET) return KASCADE_OK;
  int ok = 1;
  KS_TRY(check_is_list(ctx, succ, n, &ok, s));
  return ok ? KASCADE_OK : KASCADE_ERR_NOT_A_LIST;
}

template <class T>
kascade_status copy_in(kascade_ctx& ctx, const T* host, uint64_t n, T** dev, cudaStream_t s) {
  *dev = nullptr;
  if (!host) return KASCADE_OK;
  *dev = alloc<T>(ctx, n);
  if (!*dev) return KASCADE_ERR_OOM;
  KS_CUDA(cudaMemcpyAsync(*dev, host, n * sizeof(T), cudaMemcpyHostToDevice, s));
  return KASCADE_OK;
}

}  // namespace

extern "C" {

KASCADE_API const char* kascade_version(void) { return "kascade_b200 0.1.0 (sm_100a)"; }

KASCADE_API const char* kascade_status_string(kascade_status s) {
  switch (s) {
    case KASCADE_OK: return "ok";
    case KASCADE_ERR_INVALID_ARG: return "invalid argument";
    case KASCADE_ERR_OUT_OF_RANGE: return "successor or parent index out of range";
    case KASCADE_ERR_CYCLE: return "cycle without a root";
    case KASCADE_ERR_NOT_A_LIST: return "element with two predecessors given to a list ranker";
    case KASCADE_ERR_TIMEOUT: return "bounded device wait ran out";
    case KASCADE_ERR_OOM: return "out of memory";
    case KASCADE_ERR_CUDA: return "CUDA runtime error";
    case KASCADE_ERR_TOO_LARGE: return "input larger than the supported index range";
    case KASCADE_ERR_UNSUPPORTED: return "unsupported option";
  }
  return "unknown status";
}

KASCADE_API void kascade_opts_init(kascade_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->struct_size = sizeof(kascade_opts);
  o->algorithm = KASCADE_ALGO_SPARSE_RULING_SET;
}

KASCADE_API kascade_status kascade_ctx_create(int device, kascade_ctx** out) {
  if (!out) return KASCADE_ERR_INVALID_ARG;
  *out = nullptr;
  int count = 0;
  KS_CUDA(cudaGetDeviceCount(&count));
  if (device < 0 || device >= count) return KASCADE_ERR_INVALID_ARG;
  KS_CUDA(ensure_device(device));
  kascade_ctx* c = new (std::nothrow) kascade_ctx();
  if (!c) return KASCADE_ERR_OOM;
  c->device = device;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) {
    c->sm_count = prop.multiProcessorCount;
    c->l2_bytes = prop.l2CacheSize;
    c->smem_optin = prop.sharedMemPerBlockOptin;
  }
  if (cudaMalloc(&c->d_status, sizeof(DevStatus)) != cudaSuccess ||
      cudaMallocHost(&c->h_pinned, sizeof(unsigned long long) * KS_PINNED_WORDS) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->done_event, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    kascade_ctx_destroy(c);
    return KASCADE_ERR_OOM;
  }
  cudaMemset(c->d_status, 0, sizeof(DevStatus));
  *out = c;
  return KASCADE_OK;
}

KASCADE_API kascade_status kascade_ctx_destroy(kascade_ctx* c) {
  if (!c) return KASCADE_OK;
  ensure_device(c->device);
  cudaDeviceSynchronize();
  for (auto& b : c->blocks)
    if (b.owned) cudaFree(b.ptr);
  for (auto& p : c->pending) {
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  for (auto e : c->event_pool) cudaEventDestroy(e);
  if (c->done_event) cudaEventDestroy(c->done_event);
  if (c->d_status) cudaFree(c->d_status);
  if (c->h_pinned) cudaFreeHost(c->h_pinned);
  cudaGetLastError();
  delete c;
  return KASCADE_OK;
}

KASCADE_API kascade_status kascade_ctx_reserve(kascade_ctx* c, uint64_t bytes) {
  if (!c) return KASCADE_ERR_INVALID_ARG;
  KS_CUDA(ensure_device(c->device));
  KS_CUDA(cudaDeviceSynchronize());
  size_t have = 0;
  for (auto& b : c->blocks) have += b.cap;
  c->reserve_bytes = bytes;
  if (have >= bytes && c->blocks.size() == 1) return KASCADE_OK;
  for (auto& b : c->blocks)
    if (b.owned) cudaFree(b.ptr);
  c->blocks.clear();
  char* p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return KASCADE_ERR_OOM;
  }
  c->blocks.push_back({p, (size_t)bytes, 0});
  return KASCADE_OK;
}

KASCADE_API uint64_t kascade_scratch_bytes_rank_list(uint64_t n) {
  // level-0 records (16n) + ruler list (4n) + write-free path: log (16n,
  // reused by the second partition pass), window partition (16n rounded up
  // to whole 2^20-element windows), a margin of n, level-1 records/results
  // and deeper levels + per-warp log chunks, cursors and window rounding
  return 16 * n + 4 * n + 16 * n + 16 * n + n + (40 * n) / 16 + (192ull << 20);
}

KASCADE_API uint64_t kascade_scratch_bytes_root_forest(uint64_t n) {
  // tour records on 2n slots (32n) + ruler list (8n) + child lists, packed
  // parents and bit tables (~13n) + write-free level 0 over the <= 2n tour
  // elements: log (32n), first-pass windows (16n) + deeper levels, with
  // headroom
  return 16 * n + 8 * n + 32 * n + 8 * n + 32 * n + 16 * n + (80 * n) / 16 + (192ull << 20);
}

kascade_status rank_list_host_call(kascade_ctx* c, const uint64_t* succ, const uint32_t* weights, uint64_t n,
                                   uint64_t* root_out, uint64_t* rank_out, const kascade_opts* opts,
                                   cudaStream_t s, bool dev);
kascade_status root_forest_host_call(kascade_ctx* c, const uint64_t* parent, uint64_t n, uint64_t* root_out,
                                     uint64_t* depth_out, const kascade_opts* opts, cudaStream_t s, bool dev);

KASCADE_API kascade_status kascade_ctx_sync(kascade_ctx* c, void* stream) {
  if (!c) return KASCADE_ERR_INVALID_ARG;
  if (!c->async_pending) return c->last_status;
  c->async_pending = false;
  kascade_status st = status_finish(*c, as_stream(stream));
  if (st == KASCADE_ERR_TIMEOUT && c->host_rerun.set) {
    // an async host-buffer call whose level outgrew the device-driven
    // recursion: rank it again, on the host-driven path, before returning
    const kascade_ctx::HostRerun r = c->host_rerun;
    kascade_opts o = r.opts;
    o.async = 0;
    st = r.kind == 0 ? rank_list_host_call(c, r.succ, r.weights, r.n, r.root_out, r.rank_out, &o, r.stream, false)
                     : root_forest_host_call(c, r.succ, r.n, r.root_out, r.rank_out, &o, r.stream, false);
  }
  c->host_rerun.set = false;
  return st;
}

KASCADE_API uint64_t kascade_ctx_error_info(kascade_ctx* c) { return c ? c->error_info : 0; }

KASCADE_API int kascade_ctx_kernel_times(kascade_ctx* c, const char** names, double* ms, uint64_t* launches, int cap) {
  if (!c) return 0;
  c->time_names.clear();
  for (auto& kv : c->times) c->time_names.push_back(kv.first);
  int i = 0;
  for (auto& kv : c->times) {
    if (i >= cap) break;
    if (names) names[i] = c->time_names[i].c_str();
    if (ms) ms[i] = kv.second.first;
    if (launches) launches[i] = kv.second.second;
    ++i;
  }
  return (int)c->times.size();
}

KASCADE_API void kascade_ctx_reset_kernel_times(kascade_ctx* c) {
  if (c) c->times.clear();
}

KASCADE_API int kascade_ctx_last_levels(kascade_ctx* c, uint64_t* sizes, int cap) {
  if (!c) return 0;
  int n = (int)c->last_levels.size();
  for (int i = 0; i < n && i < cap; ++i) sizes[i] = c->last_levels[i];
  return n;
}

KASCADE_API kascade_status kascade_rank_list(kascade_ctx* c, const uint64_t* succ, const uint32_t* weights, uint64_t n,
                                             uint64_t* root_out, uint64_t* rank_out, const kascade_opts* opts,
                                             void* stream) {
  cudaStream_t s = as_stream(stream);
  if (n && (!succ || !root_out || !rank_out)) return KASCADE_ERR_INVALID_ARG;
  const bool dev = !(opts && opts->async);  // an async call's status is read later: no rerun
  KS_TRY(begin_call(c, s, opts));
  Params p = make_params(*c, opts, n);
  kascade_status st = validate_list(*c, succ, n, opts, p, s);
  if (st == KASCADE_OK)
    st = rank_list_generic(*c, succ, weights ? WKind::U32 : WKind::Unit, weights, n, root_out, rank_out, 0, p, s,
                           dev);
  st = end_call(c, s, st, opts);
  if (st != KASCADE_ERR_TIMEOUT || !dev) return st;
  // a level outgrew the device-driven recursion: rank again on the host-driven path
  KS_TRY(begin_call(c, s, opts));
  st = rank_list_generic(*c, succ, weights ? WKind::U32 : WKind::Unit, weights, n, root_out, rank_out, 0, p, s);
  return end_call(c, s, st, opts);
}

// The host-buffer list call: copies in, ranks (dev: with the device-driven
// recursion, no host wait inside the call), copies out.
kascade_status rank_list_host_call(kascade_ctx* c, const uint64_t* succ, const uint32_t* weights, uint64_t n,
                                   uint64_t* root_out, uint64_t* rank_out, const kascade_opts* opts,
                                   cudaStream_t s, bool dev) {
  KS_TRY(begin_call(c, s, opts));
  Params p = make_params(*c, opts, n);
  kascade_status st = KASCADE_OK;
  uint64_t *d_succ = nullptr, *d_root = nullptr, *d_rank = nullptr;
  uint32_t* d_w = nullptr;
  if (n) {
    st = copy_in(*c, succ, n, &d_succ, s);
    if (st == KASCADE_OK) st = copy_in(*c, weights, n, &d_w, s);
    if (st == KASCADE_OK) {
      d_root = alloc<uint64_t>(*c, n);
      d_rank = alloc<uint64_t>(*c, n);
      if (!d_root || !d_rank) st = KASCADE_ERR_OOM;
    }
    if (st == KASCADE_OK) st = validate_list(*c, d_succ, n, opts, p, s);
    if (st == KASCADE_OK)
      st = rank_list_generic(*c, d_succ, d_w ? WKind::U32 : WKind::Unit, d_w, n, d_root, d_rank, 0, p, s, dev);
    if (st == KASCADE_OK) {
      cudaError_t e = cudaMemcpyAsync(root_out, d_root, n * 8, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaMemcpyAsync(rank_out, d_rank, n * 8, cudaMemcpyDeviceToHost, s);
      st = cuda_status(e);
    }
  }
  // opts->async: return once enqueued; the host buffers belong to the call
  // until kascade_ctx_sync
  return end_call(c, s, st, opts);
}

KASCADE_API kascade_status kascade_rank_list_host(kascade_ctx* c, const uint64_t* succ, const uint32_t* weights,
                                                  uint64_t n, uint64_t* root_out, uint64_t* rank_out,
                                                  const kascade_opts* opts, void* stream) {
  cudaStream_t s = as_stream(stream);
  if (!c) return KASCADE_ERR_INVALID_ARG;
  if (n && (!succ || !root_out || !rank_out)) return KASCADE_ERR_INVALID_ARG;
  if (n > MAX_LIST) return KASCADE_ERR_TOO_LARGE;
  kascade_status st = rank_list_host_call(c, succ, weights, n, root_out, rank_out, opts, s, true);
  if (opts && opts->async) {
    if (st == KASCADE_OK) {
      c->host_rerun = kascade_ctx::HostRerun{true, 0, succ, weights, n, root_out, rank_out, *opts, s};
    }
    return st;
  }
  if (st != KASCADE_ERR_TIMEOUT) return st;
  // a level outgrew the device-driven recursion: copy in and rank again on
  // the host-driven path
  return rank_list_host_call(c, succ, weights, n, root_out, rank_out, opts, s, false);
}

KASCADE_API kascade_status kascade_sparse_ruling_set(kascade_ctx* c, const kascade_opts* opts, uint64_t* succ_array,
                                                     int64_t* rank_array, uint64_t n, void* stream) {
  cudaStream_t s = as_stream(stream);
  if (n && (!succ_array || !rank_array)) return KASCADE_ERR_INVALID_ARG;
  KS_TRY(begin_call(c, s, opts));
  Params p = make_params(*c, opts, n);
  p.algorithm = KASCADE_ALGO_SPARSE_RULING_SET;
  kascade_status st = KASCADE_OK;
  if (opts && opts->validate) {
    int ok = 1;
    st = check_is_list(*c, succ_array, n, &ok, s);
    if (st == KASCADE_OK && !ok) st = KASCADE_ERR_NOT_A_LIST;
  }
  if (st == KASCADE_OK)
    st = rank_list_generic(*c, succ_array, WKind::I64, rank_array, n, succ_array, (uint64_t*)rank_array, 1, p, s);
  return end_call(c, s, st, opts);
}

KASCADE_API kascade_status kascade_pointer_doubling(kascade_ctx* c, const kascade_opts* opts, uint64_t* succ_array,
                                                    int64_t* rank_array, uint64_t n, void* stream) {
  cudaStream_t s = as_stream(stream);
  if (n && (!succ_array || !rank_array)) return KASCADE_ERR_INVALID_ARG;
  KS_TRY(begin_call(c, s, opts));
  Params p = make_params(*c, opts, n);
  p.algorithm = KASCADE_ALGO_POINTER_DOUBLING;
  kascade_status st =
      rank_list_generic(*c, succ_array, WKind::I64, rank_array, n, succ_array, (uint64_t*)rank_array, 1, p, s);
  return end_call(c, s, st, opts);
}

KASCADE_API kascade_status kascade_rank_on_root(kascade_ctx* c, uint64_t* succ_array, int64_t* rank_array, uint64_t n,
                                                void* stream) {
  kascade_opts o;
  kascade_opts_init(&o);
  o.algorithm = KASCADE_ALGO_GATHER_CHASE;
  return kascade_pointer_doubling(c, &o, succ_array, rank_array, n, stream);
}

KASCADE_API kascade_status kascade_set_initial_ranking_state(kascade_ctx* c, const uint64_t* succ, uint64_t* root_array,
                                                             int64_t* rank_array, uint64_t n, void* stream) {
  cudaStream_t s = as_stream(stream);
  if (n && (!succ || !root_array || !rank_array)) return KASCADE_ERR_INVALID_ARG;
  KS_TRY(begin_call(c, s, nullptr));
  kascade_status st = initial_state(*c, succ, n, root_array, rank_array, s);
  return end_call(c, s, st, nullptr);
}

KASCADE_API kascade_status kascade_is_list(kascade_ctx* c, const uint64_t* succ, uint64_t n, int* is_list_out,
                                           void* stream) {
  cudaStream_t s = as_stream(stream);
  if (!is_list_out || (n && !succ)) return KASCADE_ERR_INVALID_ARG;
  *is_list_out = 1;
  KS_TRY(begin_call(c, s, nullptr));
  kascade_status st = n ? check_is_list(*c, succ, n, is_list_out, s) : KASCADE_OK;
  return end_call(c, s, st, nullptr);
}

KASCADE_API kascade_status kascade_compute_stats(kascade_ctx* c, const uint64_t* root, const int64_t* rank, uint64_t n,
                                                 int level, kascade_stats* out, kascade_tree_stats* per_tree,
                                                 uint64_t per_tree_cap, uint64_t* per_tree_count, void* stream) {
  cudaStream_t s = as_stream(stream);
  if (!out || (n && (!root || !rank)) || level < KASCADE_STATS_NONE || level > KASCADE_STATS_EXTENSIVE)
    return KASCADE_ERR_INVALID_ARG;
  std::memset(out, 0, sizeof(*out));
  if (per_tree_count) *per_tree_count = 0;
  if (level == KASCADE_STATS_NONE || n == 0) return KASCADE_OK;
  KS_TRY(begin_call(c, s, nullptr));
  kascade_status st =
      compute_stats(*c, root, rank, n, level, out, per_tree, per_tree_cap, per_tree_count, s);
  return end_call(c, s, st, nullptr);
}

KASCADE_API kascade_status kascade_root_forest(kascade_ctx* c, const uint64_t* parent, uint64_t n, uint64_t* root_out,
                                               uint64_t* depth_out, const kascade_opts* opts, void* stream) {
  cudaStream_t s = as_stream(stream);
  if (n && (!parent || !root_out || !depth_out)) return KASCADE_ERR_INVALID_ARG;
  if (n > MAX_FOREST) return KASCADE_ERR_TOO_LARGE;
  const bool dev = !(opts && opts->async);
  KS_TRY(begin_call(c, s, opts));
  Params p = make_params(*c, opts, 2 * n);
  p.algorithm = KASCADE_ALGO_SPARSE_RULING_SET;
  kascade_status st = root_forest_impl(*c, parent, (uint32_t)n, root_out, depth_out, 0, p, s, dev);
  st = end_call(c, s, st, opts);
  if (st != KASCADE_ERR_TIMEOUT || !dev) return st;
  // a tour level outgrew the device-driven recursion: again on the host-driven path
  KS_TRY(begin_call(c, s, opts));
  st = root_forest_impl(*c, parent, (uint32_t)n, root_out, depth_out, 0, p, s);
  return end_call(c, s, st, opts);
}

// The host-buffer forest call: copies in, roots (dev: with the device-driven
// recursion, no host wait inside the call), copies out.
kascade_status root_forest_host_call(kascade_ctx* c, const uint64_t* parent, uint64_t n, uint64_t* root_out,
                                     uint64_t* depth_out, const kascade_opts* opts, cudaStream_t s, bool dev) {
  KS_TRY(begin_call(c, s, opts));
  Params p = make_params(*c, opts, 2 * n);
  p.algorithm = KASCADE_ALGO_SPARSE_RULING_SET;
  kascade_status st = KASCADE_OK;
  if (n) {
    uint64_t *d_par = nullptr, *d_root = nullptr, *d_depth = nullptr;
    st = copy_in(*c, parent, n, &d_par, s);
    if (st == KASCADE_OK) {
      d_root = alloc<uint64_t>(*c, n);
      d_depth = alloc<uint64_t>(*c, n);
      if (!d_root || !d_depth) st = KASCADE_ERR_OOM;
    }
    if (st == KASCADE_OK) st = root_forest_impl(*c, d_par, (uint32_t)n, d_root, d_depth, 0, p, s, dev);
    if (st == KASCADE_OK) {
      cudaError_t e = cudaMemcpyAsync(root_out, d_root, n * 8, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaMemcpyAsync(depth_out, d_depth, n * 8, cudaMemcpyDeviceToHost, s);
      st = cuda_status(e);
    }
  }
  // opts->async: return once enqueued; the host buffers belong to the call
  // until kascade_ctx_sync
  return end_call(c, s, st, opts);
}

KASCADE_API kascade_status kascade_root_forest_host(kascade_ctx* c, const uint64_t* parent, uint64_t n,
                                                    uint64_t* root_out, uint64_t* depth_out, const kascade_opts* opts,
                                                    void* stream) {
  cudaStream_t s = as_stream(stream);
  if (!c) return KASCADE_ERR_INVALID_ARG;
  if (n && (!parent || !root_out || !depth_out)) return KASCADE_ERR_INVALID_ARG;
  if (n > MAX_FOREST) return KASCADE_ERR_TOO_LARGE;
  kascade_status st = root_forest_host_call(c, parent, n, root_out, depth_out, opts, s, true);
  if (opts && opts->async) {
    if (st == KASCADE_OK)
      c->host_rerun = kascade_ctx::HostRerun{true, 1, parent, nullptr, n, root_out, depth_out, *opts, s};
    return st;
  }
  if (st != KASCADE_ERR_TIMEOUT) return st;
  // a tour level outgrew the device-driven recursion: copy in and root again
  // on the host-driven path
  return root_forest_host_call(c, parent, n, root_out, depth_out, opts, s, false);
}

KASCADE_API kascade_status kascade_rank_via_euler_tour(kascade_ctx* c, const kascade_opts* opts, uint64_t* succ_array,
                                                       int64_t* rank_array, uint64_t n, void* stream) {
  cudaStream_t s = as_stream(stream);
  if (n && (!succ_array || !rank_array)) return KASCADE_ERR_INVALID_ARG;
  if (n > MAX_FOREST) return KASCADE_ERR_TOO_LARGE;
  KS_TRY(begin_call(c, s, opts));
  Params p = make_params(*c, opts, 2 * n);
  p.algorithm = KASCADE_ALGO_SPARSE_RULING_SET;
  kascade_status st = KASCADE_OK;
  if (n) {
    // the parent array is read by the sort before any output is written, but
    // the tour build reads it no more; results go straight to the arrays
    uint64_t* parent_copy = alloc<uint64_t>(*c, n);
    if (!parent_copy) st = KASCADE_ERR_OOM;
    if (st == KASCADE_OK)
      st = cuda_status(cudaMemcpyAsync(parent_copy, succ_array, n * 8, cudaMemcpyDeviceToDevice, s));
    if (st == KASCADE_OK)
      st = root_forest_impl(*c, parent_copy, (uint32_t)n, succ_array, (uint64_t*)rank_array, 1, p, s);
  }
  return end_call(c, s, st, opts);
}

KASCADE_API kascade_status kascade_compute_euler_tour(kascade_ctx* c, const uint64_t* parent, uint64_t n,
                                                      uint64_t* tour_succ, uint64_t* m_out, void* stream) {
  cudaStream_t s = as_stream(stream);
  if (!m_out || (n && (!parent || !tour_succ))) return KASCADE_ERR_INVALID_ARG;
  if (n > MAX_FOREST) return KASCADE_ERR_TOO_LARGE;
  *m_out = 0;
  KS_TRY(begin_call(c, s, nullptr));
  kascade_status st = compute_euler_tour_impl(*c, parent, (uint32_t)n, tour_succ, m_out, s);
  return end_call(c, s, st, nullptr);
}

KASCADE_API kascade_status kascade_pack(kascade_ctx* c, const uint64_t* succ, const int64_t* rank, uint64_t n,
                                        const uint64_t* active, uint64_t k, uint64_t* succ_packed,
                                        int64_t* rank_packed, void* stream) {
  cudaStream_t s = as_stream(stream);
  if (k > n || (k && (!succ || !rank || !active || !succ_packed || !rank_packed))) return KASCADE_ERR_INVALID_ARG;
  KS_TRY(begin_call(c, s, nullptr));
  kascade_status st = pack_impl(*c, succ, rank, n, active, k, succ_packed, rank_packed, s);
  return end_call(c, s, st, nullptr);
}

KASCADE_API kascade_status kascade_unpack(kascade_ctx* c, const uint64_t* succ_packed, const int64_t* rank_packed,
                                          const uint64_t* active, uint64_t k, uint64_t* succ, int64_t* rank,
                                          uint64_t n, void* stream) {
  cudaStream_t s = as_stream(stream);
  if (k > n || (k && (!succ || !rank || !active || !succ_packed || !rank_packed))) return KASCADE_ERR_INVALID_ARG;
  KS_TRY(begin_call(c, s, nullptr));
  kascade_status st = unpack_impl(*c, succ_packed, rank_packed, active, k, succ, rank, n, s);
  return end_call(c, s, st, nullptr);
}

KASCADE_API kascade_status kascade_rank_batch(kascade_ctx* c, const kascade_segment* segs, uint32_t num_segs,
                                              const uint64_t* input, const uint32_t* weights, uint64_t total_n,
                                              uint64_t* root_out, uint64_t* rank_out, const kascade_opts* opts,
                                              void* stream) {
  cudaStream_t s = as_stream(stream);
  if (total_n && (!segs || !num_segs || !input || !root_out || !rank_out)) return KASCADE_ERR_INVALID_ARG;
  // The device-driven recursion (no host waits) first; a batch it cannot hold
  // (a level outgrowing its capacity, e.g. very many roots) reports
  // KASCADE_ERR_TIMEOUT and is ranked again on the host-driven path.  Async
  // calls take the host-driven path directly (their status is read later).
  const bool async = opts && opts->async;
  KS_TRY(begin_call(c, s, opts));
  kascade_status st = rank_batch_impl(*c, segs, num_segs, input, weights, total_n, root_out, rank_out, opts, s, !async);
  st = end_call(c, s, st, opts);
  if (st != KASCADE_ERR_TIMEOUT || async) return st;
  KS_TRY(begin_call(c, s, opts));
  st = rank_batch_impl(*c, segs, num_segs, input, weights, total_n, root_out, rank_out, opts, s, false);
  return end_call(c, s, st, opts);
}

extern "C++" {
namespace ks {
kascade_status rank_batch_device_call(kascade_ctx* c, const kascade_segment* segs, uint32_t nseg, const uint64_t* in,
                                      const uint32_t* weights, uint64_t total, uint64_t* root_out,
                                      uint64_t* rank_out, const kascade_opts* opts, cudaStream_t s) {
  KS_TRY(begin_call(c, s, opts));
  const kascade_status st = rank_batch_impl(*c, segs, nseg, in, weights, total, root_out, rank_out, opts, s, true);
  return end_call(c, s, st, opts);
}
kascade_status batch_plan_create(int device, const kascade_segment* segs, uint32_t nseg, const uint64_t* in,
                                 const uint32_t* weights, uint64_t total, uint64_t* root_out, uint64_t* rank_out,
                                 const kascade_opts* opts, kascade_batch_plan** out);
kascade_status batch_plan_launch(kascade_batch_plan* plan, cudaStream_t s);
}  // namespace ks
}  // extern "C++"

KASCADE_API kascade_status kascade_batch_plan_create(int device, const kascade_segment* segs, uint32_t num_segs,
                                                     const uint64_t* input, const uint32_t* weights, uint64_t total_n,
                                                     uint64_t* root_out, uint64_t* rank_out,
                                                     const kascade_opts* opts, kascade_batch_plan** plan) {
  if (!plan) return KASCADE_ERR_INVALID_ARG;
  return batch_plan_create(device, segs, num_segs, input, weights, total_n, root_out, rank_out, opts, plan);
}

KASCADE_API kascade_status kascade_batch_plan_launch(kascade_batch_plan* plan, void* stream) {
  return batch_plan_launch(plan, as_stream(stream));
}

KASCADE_API kascade_status kascade_ctx_set_size_classes(kascade_ctx* c, const uint64_t* max_size,
                                                        const uint32_t* spacing, uint32_t count) {
  if (!c || !max_size || !spacing || count == 0 || count > 64) return KASCADE_ERR_INVALID_ARG;
  for (uint32_t i = 0; i < count; ++i) {
    if (spacing[i] < 2 || (i && max_size[i] <= max_size[i - 1])) return KASCADE_ERR_INVALID_ARG;
  }
  c->class_max.assign(max_size, max_size + count);
  c->class_max.back() = ~0ull;
  c->class_spacing.assign(spacing, spacing + count);
  c->class_chains.assign(count, 2u);
  c->class_block.assign(count, 256u);
  c->class_spacing_single.assign(spacing, spacing + count);
  return KASCADE_OK;
}

KASCADE_API kascade_status kascade_ctx_set_class_launch(kascade_ctx* c, const uint32_t* chains, const uint32_t* block,
                                                        const uint32_t* single_spacing, uint32_t count) {
  if (!c || !chains || !block || count != c->class_max.size()) return KASCADE_ERR_INVALID_ARG;
  for (uint32_t i = 0; i < count; ++i) {
    if (chains[i] != 1 && chains[i] != 2 && chains[i] != 4) return KASCADE_ERR_INVALID_ARG;
    if (block[i] != 128 && block[i] != 256 && block[i] != 512) return KASCADE_ERR_INVALID_ARG;
    if (single_spacing && single_spacing[i] < 2) return KASCADE_ERR_INVALID_ARG;
  }
  c->class_chains.assign(chains, chains + count);
  c->class_block.assign(block, block + count);
  if (single_spacing) c->class_spacing_single.assign(single_spacing, single_spacing + count);
  return KASCADE_OK;
}

KASCADE_API int kascade_ctx_get_class_launch(kascade_ctx* c, uint32_t* chains, uint32_t* block,
                                             uint32_t* single_spacing, int cap) {
  if (!c) return 0;
  const int n = (int)c->class_max.size();
  for (int i = 0; i < n && i < cap; ++i) {
    if (chains) chains[i] = c->class_chains[i];
    if (block) block[i] = c->class_block[i];
    if (single_spacing) single_spacing[i] = c->class_spacing_single[i];
  }
  return n;
}

KASCADE_API kascade_status kascade_ctx_set_sm_budget(kascade_ctx* c, int sms) {
  if (!c || sms < 0) return KASCADE_ERR_INVALID_ARG;
  c->sm_budget.store(sms, std::memory_order_relaxed);
  return KASCADE_OK;
}

KASCADE_API int kascade_ctx_get_size_classes(kascade_ctx* c, uint64_t* max_size, uint32_t* spacing, int cap) {
  if (!c) return 0;
  const int n = (int)c->class_max.size();
  for (int i = 0; i < n && i < cap; ++i) {
    if (max_size) max_size[i] = c->class_max[i];
    if (spacing) spacing[i] = c->class_spacing[i];
  }
  return n;
}

KASCADE_API kascade_status kascade_gen_list(uint64_t n, uint64_t seed, uint32_t layout, uint64_t* succ, void* stream) {
  if (n && !succ) return KASCADE_ERR_INVALID_ARG;
  if (layout > KS_LAYOUT_IDENTITY) return KASCADE_ERR_INVALID_ARG;
  return gen_list(n, seed, layout, succ, as_stream(stream));
}

KASCADE_API kascade_status kascade_gen_weights(uint64_t n, uint64_t seed, uint32_t wbits, uint32_t* weights,
                                               void* stream) {
  if (n && !weights) return KASCADE_ERR_INVALID_ARG;
  if (wbits == 0 || wbits > 32) return KASCADE_ERR_INVALID_ARG;
  return gen_weights(n, seed, wbits, weights, as_stream(stream));
}

KASCADE_API kascade_status kascade_gen_forest(uint64_t n, uint64_t seed, uint32_t kind, uint64_t blocks,
                                              uint64_t spine, uint64_t* parent, void* stream) {
  if (n && !parent) return KASCADE_ERR_INVALID_ARG;
  if (kind > KS_FOREST_CATERPILLAR || blocks == 0 || (n && blocks > n)) return KASCADE_ERR_INVALID_ARG;
  return gen_forest(n, seed, kind, blocks, spine, parent, as_stream(stream));
}

}  // extern "C"
