// Batched ranking: thousands of independent lists and forests of uneven size
// ranked together.
//
// The instances arrive concatenated (instance-local indices) with a segment
// table.  They are laid out in one record space so that a single ruler chase
// -- one persistent launch with one device work queue -- serves every
// instance:
//   list element g (concatenated position)  -> record g
//   forest vertex g                         -> record g (its up edge / tour end;
//                                              a leaf's down and up edge in one)
//   down edges of all forests (F of them)   -> records total_n .. total_n+F-1
//                                              (a leaf's or a root's: a dead self loop)
// Each instance's ruler spacing comes from its size class (the context's
// size-class table, filled by the autotuner).  Roots are reported relative to
// their own instance.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "ranker.cuh"

namespace ks {

kascade_status batch_tours(kascade_ctx& ctx, const uint64_t* fpar, uint32_t F, const uint32_t* fd, const uint32_t* foff,
                           const uint32_t* fthresh, const uint32_t* fhint, uint32_t nf, uint32_t down_base, Rec* rec,
                           uint32_t* ruler_elem, uint32_t* counter, uint32_t* leaf_out, uint32_t salt,
                           cudaStream_t s);

namespace {

constexpr uint32_t ITEM = 4096;  // elements per work item
constexpr int BP_THREADS = 256;
constexpr int BP_PER = ITEM / BP_THREADS;

struct __align__(16) DSeg {
  unsigned long long off;
  uint32_t size;
  uint32_t kind;
  uint32_t thresh;
  uint32_t fd;  // forests: base in the compact forest vertex space
};

struct __align__(16) Item {
  uint32_t seg;
  uint32_t start;
  uint32_t count;
  uint32_t pad;
};

struct BWUnit {
  __device__ __forceinline__ uint64_t operator()(uint64_t) const { return 1ull; }
};
struct BWU32 {
  const uint32_t* p;
  __device__ __forceinline__ uint64_t operator()(uint64_t g) const { return (uint64_t)__ldcs(p + g); }
};

template <class W>
__global__ void __launch_bounds__(BP_THREADS) k_batch_prepare(const Item* __restrict__ items, uint32_t nitems,
                                                              const DSeg* __restrict__ segs,
                                                              const uint64_t* __restrict__ in, W w,
                                                              Rec* __restrict__ rec, uint64_t* __restrict__ fpar,
                                                              uint32_t* __restrict__ ruler_elem,
                                                              uint32_t* __restrict__ counter, uint32_t salt,
                                                              DevStatus* st) {
  __shared__ uint32_t sm[33];
  __shared__ uint32_t sbase;
  for (uint32_t it = blockIdx.x; it < nitems; it += gridDim.x) {
    const Item item = items[it];
    const DSeg sg = segs[item.seg];
    if (sg.kind == KASCADE_SEG_LIST) {
      uint32_t sv[BP_PER];
      uint64_t wv[BP_PER];
      unsigned long long lv[BP_PER];
      uint32_t rl = 0, cnt = 0;
      // every load of the item first (independent, all in flight together),
      // then the checks and the sampling
#pragma unroll
      for (int i = 0; i < BP_PER; ++i) {
        const uint32_t k = item.start + i * BP_THREADS + threadIdx.x;
        lv[i] = 0;
        wv[i] = 0;
        if (k < item.start + item.count) {
          const uint64_t g = sg.off + k;
          lv[i] = __ldcs(reinterpret_cast<const unsigned long long*>(in) + g);
          wv[i] = w(g);
        }
      }
      uint64_t bad = ~0ull;  // the first element whose successor is out of its instance
#pragma unroll
      for (int i = 0; i < BP_PER; ++i) {
        const uint32_t k = item.start + i * BP_THREADS + threadIdx.x;
        sv[i] = 0;
        if (k < item.start + item.count) {
          const uint64_t g = sg.off + k;
          unsigned long long loc = lv[i];
          if (loc >= sg.size) {
            if (bad == ~0ull) bad = g;
            loc = k;
          }
          sv[i] = (uint32_t)(sg.off + loc);
          if (loc == k || sampled((uint32_t)g, salt, sg.thresh)) {
            rl |= 1u << i;
            cnt++;
          }
        }
      }
      if (bad != ~0ull) set_error(st, KASCADE_ERR_OUT_OF_RANGE, bad);
      uint32_t total;
      const uint32_t pre = block_exclusive_scan(cnt, sm, &total);
      if (threadIdx.x == 0) {
        const uint32_t b = total ? atomicAdd(counter, total) : 0u;
        if ((uint64_t)b + total > MAX_RULERS) set_error(st, KASCADE_ERR_TOO_LARGE, b);
        sbase = b;
      }
      __syncthreads();
      uint32_t id = sbase + pre;
#pragma unroll
      for (int i = 0; i < BP_PER; ++i) {
        const uint32_t k = item.start + i * BP_THREADS + threadIdx.x;
        if (k >= item.start + item.count) continue;
        const uint32_t g = (uint32_t)(sg.off + k);
        Rec r;
        r.a = wv[i];
        r.b = sv[i];
        r.c = TAG_UNREACHED;
        if (rl & (1u << i)) {
          if (id < MAX_RULERS) {
            r.c = TAG_RULER | id;
            ruler_elem[id] = g;
          }
          id++;
        }
        rec[g] = r;
      }
      __syncthreads();
    } else {
      unsigned long long pv[BP_PER];
#pragma unroll
      for (int i = 0; i < BP_PER; ++i) {
        const uint32_t k = item.start + i * BP_THREADS + threadIdx.x;
        pv[i] = k < item.start + item.count ? __ldcs(reinterpret_cast<const unsigned long long*>(in) + sg.off + k) : 0;
      }
      uint64_t bad = ~0ull;
#pragma unroll
      for (int i = 0; i < BP_PER; ++i) {
        const uint32_t k = item.start + i * BP_THREADS + threadIdx.x;
        if (k >= item.start + item.count) continue;
        unsigned long long par = pv[i];
        if (par >= sg.size) {
          if (bad == ~0ull) bad = sg.off + k;
          par = k;
        }
        __stcs(reinterpret_cast<unsigned long long*>(fpar) + sg.fd + k, (unsigned long long)(sg.fd + par));
      }
      if (bad != ~0ull) set_error(st, KASCADE_ERR_OUT_OF_RANGE, bad);
    }
  }
}

inline uint32_t thresh_of(uint32_t spacing) {
  if (spacing <= 1) return 0xFFFFFFFFu;
  const double t = 4294967296.0 / (double)spacing;
  return t >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)t;
}

}  // namespace

constexpr uint32_t WRITE_FREE_MIN_SPACING = 48;

uint32_t spacing_for(const kascade_ctx& ctx, uint64_t n) {
  for (size_t i = 0; i < ctx.class_max.size(); ++i)
    if (n <= ctx.class_max[i]) return ctx.class_spacing[i];
  return ctx.class_spacing.empty() ? 48u : ctx.class_spacing.back();
}

// Host tables of one batch: built from the segment list, uploaded into the
// context's arena.  Kept apart from the launches so that a plan can upload
// them once and capture only the device work.
struct BatchTables {
  std::vector<DSeg> dsegs;
  std::vector<Item> items;
  std::vector<uint32_t> fd, foff, fth, hint, fhint;
  std::vector<unsigned long long> seg_off;
  uint64_t total = 0, F = 0;
  uint32_t nseg = 0, nf = 0, M = 0, spacing_min = 0xFFFFFFFFu, spacing_max = 0;
  size_t dom_class = 0;  // the size class holding most of the batch's records
  // device copies
  DSeg* d_segs = nullptr;
  Item* d_items = nullptr;
  uint32_t *d_fd = nullptr, *d_foff = nullptr, *d_fth = nullptr, *d_hint = nullptr, *d_fhint = nullptr;
  unsigned long long* d_off = nullptr;
};

kascade_status batch_build_tables(const kascade_ctx& ctx, const kascade_segment* segs, uint32_t nseg, uint64_t total,
                                  const kascade_opts* opts, BatchTables& t) {
  t = BatchTables{};
  t.nseg = nseg;
  t.total = total;
  t.dsegs.resize(nseg);
  t.seg_off.resize(nseg);
  std::vector<uint64_t> class_elems(ctx.class_max.size(), 0);
  t.items.reserve(total / ITEM + nseg);
  // A batch large enough for the write-free level 0 samples its rulers more
  // sparsely: its chase is read-only and cheap per hop, so fewer rulers (a
  // smaller recursion) pay off.  Measured on the 4096-instance, 2^28-element
  // batch: class spacings (4-24) 34.2 ms, a floor of 16 28.0, 32 27.2, 48
  // 27.0 ms, results identical.
  uint32_t spacing_floor = 0;
  if (!(opts && opts->ruler_spacing)) {
    uint64_t records = total;
    for (uint32_t i = 0; i < nseg; ++i)
      if (segs[i].kind == KASCADE_SEG_FOREST) records += segs[i].size;
    const Params pm = make_params(ctx, opts, records);
    if (records >= pm.level0_log_min && pm.max_levels > 0 && records > pm.base_max)
      spacing_floor = WRITE_FREE_MIN_SPACING;
  }
  uint64_t expect = 0;
  for (uint32_t i = 0; i < nseg; ++i) {
    const kascade_segment& g = segs[i];
    if (g.offset != expect || g.size > 0x7FFFFFFFull || (g.kind != KASCADE_SEG_LIST && g.kind != KASCADE_SEG_FOREST))
      return KASCADE_ERR_INVALID_ARG;
    expect += g.size;
    const bool forest = g.kind == KASCADE_SEG_FOREST;
    const uint64_t records = forest ? 2 * g.size : g.size;
    const uint32_t spacing =
        (opts && opts->ruler_spacing) ? opts->ruler_spacing : std::max(spacing_for(ctx, records), spacing_floor);
    class_elems[ctx.class_of(records)] += records;
    if (g.size) {
      t.spacing_min = std::min(t.spacing_min, spacing);
      t.spacing_max = std::max(t.spacing_max, spacing);
    }
    t.dsegs[i] = DSeg{g.offset, (uint32_t)g.size, g.kind, thresh_of(spacing), (uint32_t)t.F};
    t.seg_off[i] = g.offset;
    if (forest) {
      t.fd.push_back((uint32_t)t.F);
      t.foff.push_back((uint32_t)g.offset);
      t.fth.push_back(thresh_of(spacing));
      t.F += g.size;
    }
    for (uint64_t st = 0; st < g.size; st += ITEM)
      t.items.push_back(Item{i, (uint32_t)st, (uint32_t)std::min<uint64_t>(ITEM, g.size - st), 0});
  }
  if (expect != total) return KASCADE_ERR_INVALID_ARG;
  if (total + t.F > MAX_ELEMS) return KASCADE_ERR_TOO_LARGE;
  t.nf = (uint32_t)t.fd.size();
  t.fd.push_back((uint32_t)t.F);
  t.hint.resize((size_t)((total + 4095) / 4096) + 1);
  {
    uint32_t j = 0;
    for (size_t k = 0; k < t.hint.size(); ++k) {
      const uint64_t x = (uint64_t)k * 4096;
      while (j + 1 < nseg && t.seg_off[j + 1] <= x) ++j;
      t.hint[k] = j;
    }
  }
  // per 4096 compact forest vertices: the forest holding the first (and one
  // entry past the last block, so a block's search range is [fhint[k], fhint[k+1]])
  t.fhint.resize((size_t)((t.F + 4095) / 4096) + 1);
  {
    uint32_t j = 0;
    for (size_t k = 0; k < t.fhint.size(); ++k) {
      const uint64_t c = (uint64_t)k * 4096;
      while (j + 1 < t.nf && t.fd[j + 1] <= c) ++j;
      t.fhint[k] = j;
    }
  }
  t.M = (uint32_t)(total + t.F);
  t.dom_class = std::max_element(class_elems.begin(), class_elems.end()) - class_elems.begin();
  return KASCADE_OK;
}

kascade_status batch_upload_tables(kascade_ctx& ctx, BatchTables& t, cudaStream_t s) {
  t.d_segs = alloc<DSeg>(ctx, t.nseg);
  t.d_items = alloc<Item>(ctx, t.items.size() + 1);
  t.d_fd = alloc<uint32_t>(ctx, t.fd.size());
  t.d_foff = alloc<uint32_t>(ctx, t.foff.size() + 1);
  t.d_fth = alloc<uint32_t>(ctx, t.fth.size() + 1);
  t.d_off = alloc<unsigned long long>(ctx, t.nseg);
  t.d_hint = alloc<uint32_t>(ctx, t.hint.size());
  t.d_fhint = alloc<uint32_t>(ctx, t.fhint.size());
  if (!t.d_segs || !t.d_items || !t.d_fd || !t.d_foff || !t.d_fth || !t.d_off || !t.d_hint || !t.d_fhint)
    return KASCADE_ERR_OOM;
  KS_CUDA(cudaMemcpyAsync(t.d_segs, t.dsegs.data(), sizeof(DSeg) * t.nseg, cudaMemcpyHostToDevice, s));
  KS_CUDA(cudaMemcpyAsync(t.d_items, t.items.data(), sizeof(Item) * t.items.size(), cudaMemcpyHostToDevice, s));
  KS_CUDA(cudaMemcpyAsync(t.d_fd, t.fd.data(), sizeof(uint32_t) * t.fd.size(), cudaMemcpyHostToDevice, s));
  if (t.nf) {
    KS_CUDA(cudaMemcpyAsync(t.d_foff, t.foff.data(), sizeof(uint32_t) * t.nf, cudaMemcpyHostToDevice, s));
    KS_CUDA(cudaMemcpyAsync(t.d_fth, t.fth.data(), sizeof(uint32_t) * t.nf, cudaMemcpyHostToDevice, s));
  }
  KS_CUDA(cudaMemcpyAsync(t.d_off, t.seg_off.data(), sizeof(unsigned long long) * t.nseg, cudaMemcpyHostToDevice, s));
  KS_CUDA(cudaMemcpyAsync(t.d_hint, t.hint.data(), sizeof(uint32_t) * t.hint.size(), cudaMemcpyHostToDevice, s));
  KS_CUDA(cudaMemcpyAsync(t.d_fhint, t.fhint.data(), sizeof(uint32_t) * t.fhint.size(), cudaMemcpyHostToDevice, s));
  return KASCADE_OK;
}

// The device work of one batch over uploaded tables: no host tables are read
// and, with device_levels, no host waits -- a stream capture of this call is
// a replayable CUDA graph.
kascade_status batch_enqueue(kascade_ctx& ctx, const BatchTables& t, const uint64_t* in, const uint32_t* weights,
                             uint64_t* root_out, uint64_t* rank_out, const kascade_opts* opts, cudaStream_t s,
                             bool device_levels) {
  const uint32_t M = t.M;
  Rec* rec = alloc<Rec>(ctx, M);
  uint32_t* ruler_elem = alloc<uint32_t>(ctx, M);
  uint64_t* fpar = alloc<uint64_t>(ctx, t.F + 1);
  uint32_t* ctr = alloc<uint32_t>(ctx, 1);
  // forest leaves by output position: their rank is one less than their depth
  const uint64_t leaf_words = t.F ? (t.total + 31) / 32 : 0;
  uint32_t* leaf_out = leaf_words ? alloc<uint32_t>(ctx, leaf_words) : nullptr;
  if (!rec || !ruler_elem || !fpar || !ctr || (leaf_words && !leaf_out)) return KASCADE_ERR_OOM;
  KS_CUDA(cudaMemsetAsync(ctr, 0, sizeof(uint32_t), s));
  if (leaf_out) KS_CUDA(cudaMemsetAsync(leaf_out, 0, sizeof(uint32_t) * leaf_words, s));
  Params p = make_params(ctx, opts, M);
  {
    // one chase launch serves every instance: its chains and block size come
    // from the class that holds most of the batch's elements
    const size_t k = t.dom_class;
    if (!(opts && opts->chains_per_thread)) p.chains = ctx.class_chains[k];
    if (!(opts && opts->block_size)) p.block = (ctx.class_block[k] == 128 || ctx.class_block[k] == 512)
                                                   ? ctx.class_block[k] : 256u;
  }
  const uint32_t salt = mix32(p.seed ^ 0x62617463u);
  {
    ProfScope ps(ctx, "batch_prepare", s);
    const unsigned grid = (unsigned)std::min<uint64_t>(t.items.size(), (uint64_t)ctx.usable_sms() * 8);
    if (weights)
      k_batch_prepare<BWU32><<<grid, BP_THREADS, 0, s>>>(t.d_items, (uint32_t)t.items.size(), t.d_segs, in,
                                                         BWU32{weights}, rec, fpar, ruler_elem, ctr, salt,
                                                         ctx.d_status);
    else
      k_batch_prepare<BWUnit><<<grid, BP_THREADS, 0, s>>>(t.d_items, (uint32_t)t.items.size(), t.d_segs, in,
                                                          BWUnit{}, rec, fpar, ruler_elem, ctr, salt, ctx.d_status);
    KS_CHECK_LAUNCH();
  }
  KS_TRY(batch_tours(ctx, fpar, (uint32_t)t.F, t.d_fd, t.d_foff, t.d_fth, t.d_fhint, t.nf, (uint32_t)t.total, rec,
                     ruler_elem, ctr, leaf_out, mix32(p.seed ^ 0x70757254u), s));
  SinkBatch sink{root_out, rank_out, (uint32_t)t.total, reinterpret_cast<const uint64_t*>(t.d_off), t.d_hint, t.nseg,
                 leaf_out};
  p.algorithm = KASCADE_ALGO_SPARSE_RULING_SET;
  // the write-free chase's hop cap follows the sparsest instance's spacing
  if (!(opts && opts->max_chain)) p.max_chain = 64u * std::max(t.spacing_max, p.spacing0) + 1024u;
  if (device_levels) {
    // no host wait: the level-0 ruler count stays on the device
    if (M <= p.base_max) return rank_records(ctx, rec, M, 0u, ruler_elem, sink, p, s);
    const uint32_t cap1 = dev_cap_next(M, t.spacing_min);
    if (M >= p.level0_log_min && p.max_levels > 0)
      return rank_level0_log(ctx, rec, M, cap1, ruler_elem, sink.log_target(M), p, s, ctr);
    return rank_records_dev(ctx, rec, M, ctr, cap1, ruler_elem, sink, p, s);
  }
  uint32_t r0 = 0;
  KS_TRY(read_u32(ctx, ctr, &r0, s));
  return rank_records(ctx, rec, M, r0, ruler_elem, sink, p, s);
}

kascade_status rank_batch_impl(kascade_ctx& ctx, const kascade_segment* segs, uint32_t nseg, const uint64_t* in,
                               const uint32_t* weights, uint64_t total, uint64_t* root_out, uint64_t* rank_out,
                               const kascade_opts* opts, cudaStream_t s, bool device_levels) {
  if (total == 0) return KASCADE_OK;
  BatchTables t;
  KS_TRY(batch_build_tables(ctx, segs, nseg, total, opts, t));
  KS_TRY(batch_upload_tables(ctx, t, s));
  return batch_enqueue(ctx, t, in, weights, root_out, rank_out, opts, s, device_levels);
}

// ---------------------------------------------------------------------------
// Plans: one batch captured as a CUDA graph and replayed.
// ---------------------------------------------------------------------------
// A complete call on the device-driven path (status read back), in capi.cu.
kascade_status rank_batch_device_call(kascade_ctx* c, const kascade_segment* segs, uint32_t nseg, const uint64_t* in,
                                      const uint32_t* weights, uint64_t total, uint64_t* root_out,
                                      uint64_t* rank_out, const kascade_opts* opts, cudaStream_t s);
}  // namespace ks

struct kascade_batch_plan {
  kascade_ctx* ctx = nullptr;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace ks {

kascade_status batch_plan_create(int device, const kascade_segment* segs, uint32_t nseg, const uint64_t* in,
                                 const uint32_t* weights, uint64_t total, uint64_t* root_out, uint64_t* rank_out,
                                 const kascade_opts* opts_in, kascade_batch_plan** out) {
  *out = nullptr;
  if (total == 0 || !segs || !nseg || !in || !root_out || !rank_out) return KASCADE_ERR_INVALID_ARG;
  kascade_opts opts;
  kascade_opts_init(&opts);
  if (opts_in) std::memcpy(&opts, opts_in, std::min<size_t>(sizeof(opts), opts_in->struct_size ? opts_in->struct_size
                                                                                                : sizeof(opts)));
  opts.struct_size = sizeof(opts);
  opts.profile = 0;
  opts.async = 0;
  auto* plan = new (std::nothrow) kascade_batch_plan();
  if (!plan) return KASCADE_ERR_OOM;
  auto fail = [&](kascade_status st) {
    kascade_batch_plan_destroy(plan);
    return st;
  };
  KS_TRY(kascade_ctx_create(device, &plan->ctx));
  kascade_ctx& ctx = *plan->ctx;
  if (cudaStreamCreateWithFlags(&plan->stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    return fail(KASCADE_ERR_CUDA);
  }
  cudaStream_t s = plan->stream;
  // 1. one eager run: the batch must fit the device-driven recursion (the
  //    run also grows the plan's arena to what the batch needs)
  kascade_status st = rank_batch_device_call(plan->ctx, segs, nseg, in, weights, total, root_out, rank_out, &opts, s);
  if (st == KASCADE_ERR_TIMEOUT) return fail(KASCADE_ERR_UNSUPPORTED);
  if (st != KASCADE_OK) return fail(st);
  // 2. tables uploaded outside the capture, the device work captured
  st = arena_begin_call(ctx, s);
  BatchTables t;
  if (st == KASCADE_OK) st = batch_build_tables(ctx, segs, nseg, total, &opts, t);
  if (st == KASCADE_OK) st = batch_upload_tables(ctx, t, s);
  if (st == KASCADE_OK && cudaStreamSynchronize(s) != cudaSuccess) st = KASCADE_ERR_CUDA;
  if (st != KASCADE_OK) return fail(st);
  const size_t blocks_before = ctx.blocks.size();
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return fail(KASCADE_ERR_CUDA);
  }
  st = status_reset(ctx, s);
  if (st == KASCADE_OK) st = batch_enqueue(ctx, t, in, weights, root_out, rank_out, &opts, s, true);
  cudaGraph_t g = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(s, &g);
  plan->graph = g;
  if (st == KASCADE_OK && (ce != cudaSuccess || !g)) st = KASCADE_ERR_CUDA;
  // the capture must not have grown the arena (the eager run sized it)
  if (st == KASCADE_OK && ctx.blocks.size() != blocks_before) st = KASCADE_ERR_UNSUPPORTED;
  if (st == KASCADE_OK && cudaGraphInstantiate(&plan->exec, g, 0) != cudaSuccess) st = KASCADE_ERR_CUDA;
  cudaGetLastError();
  if (st != KASCADE_OK) return fail(st);
  *out = plan;
  return KASCADE_OK;
}

kascade_status batch_plan_launch(kascade_batch_plan* plan, cudaStream_t s) {
  if (!plan || !plan->exec) return KASCADE_ERR_INVALID_ARG;
  kascade_ctx& ctx = *plan->ctx;
  // the plan's scratch is reused by every launch: order after the previous one
  if (ctx.done_event && ctx.last_stream != s) KS_CUDA(cudaStreamWaitEvent(s, ctx.done_event, 0));
  KS_CUDA(cudaGraphLaunch(plan->exec, s));
  cudaEventRecord(ctx.done_event, s);
  ctx.last_stream = s;
  return status_finish(ctx, s);
}

}  // namespace ks

extern "C" KASCADE_API kascade_status kascade_batch_plan_destroy(kascade_batch_plan* plan) {
  if (!plan) return KASCADE_OK;
  if (plan->stream) cudaStreamSynchronize(plan->stream);
  if (plan->exec) cudaGraphExecDestroy(plan->exec);
  if (plan->graph) cudaGraphDestroy(plan->graph);
  if (plan->stream) cudaStreamDestroy(plan->stream);
  if (plan->ctx) kascade_ctx_destroy(plan->ctx);
  cudaGetLastError();
  delete plan;
  return KASCADE_OK;
}
