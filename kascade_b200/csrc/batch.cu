// Batched ranking: thousands of independent lists and forests of uneven size
// ranked together.
//
// The instances arrive concatenated (instance-local indices) with a segment
// table.  They are laid out in one record space so that a single ruler chase
// -- one persistent launch with one device work queue -- serves every
// instance:
//   list element g (concatenated position)  -> record g
//   forest vertex g                         -> record g (its up edge / tour end)
//   down edges of all forests (F of them)   -> records total_n .. total_n+F-1
// Each instance's ruler spacing comes from its size class (the context's
// size-class table, filled by the autotuner).  Roots are reported relative to
// their own instance.
#include <algorithm>
#include <vector>

#include "ranker.cuh"

namespace ks {

kascade_status batch_tours(kascade_ctx& ctx, const uint64_t* fpar, uint32_t F, const uint32_t* fd, const uint32_t* foff,
                           const uint32_t* fthresh, uint32_t nf, uint32_t down_base, Rec* rec, uint32_t* ruler_elem,
                           uint32_t* counter, uint32_t salt, cudaStream_t s);

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
      uint32_t rl = 0, cnt = 0;
#pragma unroll
      for (int i = 0; i < BP_PER; ++i) {
        const uint32_t k = item.start + i * BP_THREADS + threadIdx.x;
        sv[i] = 0;
        wv[i] = 0;
        if (k < item.start + item.count) {
          const uint64_t g = sg.off + k;
          unsigned long long loc = __ldcs(reinterpret_cast<const unsigned long long*>(in) + g);
          if (loc >= sg.size) {
            set_error(st, KASCADE_ERR_OUT_OF_RANGE, g);
            loc = k;
          }
          sv[i] = (uint32_t)(sg.off + loc);
          wv[i] = w(g);
          if (loc == k || sampled((uint32_t)g, salt, sg.thresh)) {
            rl |= 1u << i;
            cnt++;
          }
        }
      }
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
      for (uint32_t k = item.start + threadIdx.x; k < item.start + item.count; k += BP_THREADS) {
        const uint64_t g = sg.off + k;
        unsigned long long par = __ldcs(reinterpret_cast<const unsigned long long*>(in) + g);
        if (par >= sg.size) {
          set_error(st, KASCADE_ERR_OUT_OF_RANGE, g);
          par = k;
        }
        fpar[sg.fd + k] = sg.fd + par;
      }
    }
  }
}

inline uint32_t thresh_of(uint32_t spacing) {
  if (spacing <= 1) return 0xFFFFFFFFu;
  const double t = 4294967296.0 / (double)spacing;
  return t >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)t;
}

}  // namespace

uint32_t spacing_for(const kascade_ctx& ctx, uint64_t n) {
  for (size_t i = 0; i < ctx.class_max.size(); ++i)
    if (n <= ctx.class_max[i]) return ctx.class_spacing[i];
  return ctx.class_spacing.empty() ? 48u : ctx.class_spacing.back();
}

kascade_status rank_batch_impl(kascade_ctx& ctx, const kascade_segment* segs, uint32_t nseg, const uint64_t* in,
                               const uint32_t* weights, uint64_t total, uint64_t* root_out, uint64_t* rank_out,
                               const kascade_opts* opts, cudaStream_t s) {
  if (total == 0) return KASCADE_OK;
  // host tables
  std::vector<DSeg> dsegs(nseg);
  std::vector<Item> items;
  std::vector<uint32_t> fd, foff, fth;
  std::vector<unsigned long long> seg_off(nseg);
  uint64_t expect = 0, F = 0;
  std::vector<uint64_t> class_elems(ctx.class_max.size(), 0);
  items.reserve(total / ITEM + nseg);
  for (uint32_t i = 0; i < nseg; ++i) {
    const kascade_segment& g = segs[i];
    if (g.offset != expect || g.size > 0x7FFFFFFFull || (g.kind != KASCADE_SEG_LIST && g.kind != KASCADE_SEG_FOREST))
      return KASCADE_ERR_INVALID_ARG;
    expect += g.size;
    const bool forest = g.kind == KASCADE_SEG_FOREST;
    const uint64_t records = forest ? 2 * g.size : g.size;
    const uint32_t spacing = (opts && opts->ruler_spacing) ? opts->ruler_spacing : spacing_for(ctx, records);
    class_elems[ctx.class_of(records)] += records;
    dsegs[i] = DSeg{g.offset, (uint32_t)g.size, g.kind, thresh_of(spacing), (uint32_t)F};
    seg_off[i] = g.offset;
    if (forest) {
      fd.push_back((uint32_t)F);
      foff.push_back((uint32_t)g.offset);
      fth.push_back(thresh_of(spacing));
      F += g.size;
    }
    for (uint64_t st = 0; st < g.size; st += ITEM)
      items.push_back(Item{i, (uint32_t)st, (uint32_t)std::min<uint64_t>(ITEM, g.size - st), 0});
  }
  if (expect != total) return KASCADE_ERR_INVALID_ARG;
  if (total + F > MAX_ELEMS) return KASCADE_ERR_TOO_LARGE;
  const uint32_t nf = (uint32_t)fd.size();
  fd.push_back((uint32_t)F);
  std::vector<uint32_t> hint((size_t)((total + 4095) / 4096) + 1);
  {
    uint32_t j = 0;
    for (size_t k = 0; k < hint.size(); ++k) {
      const uint64_t x = (uint64_t)k * 4096;
      while (j + 1 < nseg && seg_off[j + 1] <= x) ++j;
      hint[k] = j;
    }
  }
  const uint32_t M = (uint32_t)(total + F);
  // device copies of the tables
  DSeg* d_segs = alloc<DSeg>(ctx, nseg);
  Item* d_items = alloc<Item>(ctx, items.size() + 1);
  uint32_t* d_fd = alloc<uint32_t>(ctx, fd.size());
  uint32_t* d_foff = alloc<uint32_t>(ctx, foff.size() + 1);
  uint32_t* d_fth = alloc<uint32_t>(ctx, fth.size() + 1);
  unsigned long long* d_off = alloc<unsigned long long>(ctx, nseg);
  uint32_t* d_hint = alloc<uint32_t>(ctx, hint.size());
  Rec* rec = alloc<Rec>(ctx, M);
  uint32_t* ruler_elem = alloc<uint32_t>(ctx, M);
  uint64_t* fpar = alloc<uint64_t>(ctx, F + 1);
  uint32_t* ctr = alloc<uint32_t>(ctx, 1);
  if (!d_segs || !d_items || !d_fd || !d_foff || !d_fth || !d_off || !d_hint || !rec || !ruler_elem || !fpar || !ctr)
    return KASCADE_ERR_OOM;
  KS_CUDA(cudaMemcpyAsync(d_segs, dsegs.data(), sizeof(DSeg) * nseg, cudaMemcpyHostToDevice, s));
  KS_CUDA(cudaMemcpyAsync(d_items, items.data(), sizeof(Item) * items.size(), cudaMemcpyHostToDevice, s));
  KS_CUDA(cudaMemcpyAsync(d_fd, fd.data(), sizeof(uint32_t) * fd.size(), cudaMemcpyHostToDevice, s));
  if (nf) {
    KS_CUDA(cudaMemcpyAsync(d_foff, foff.data(), sizeof(uint32_t) * nf, cudaMemcpyHostToDevice, s));
    KS_CUDA(cudaMemcpyAsync(d_fth, fth.data(), sizeof(uint32_t) * nf, cudaMemcpyHostToDevice, s));
  }
  KS_CUDA(cudaMemcpyAsync(d_off, seg_off.data(), sizeof(unsigned long long) * nseg, cudaMemcpyHostToDevice, s));
  KS_CUDA(cudaMemcpyAsync(d_hint, hint.data(), sizeof(uint32_t) * hint.size(), cudaMemcpyHostToDevice, s));
  KS_CUDA(cudaMemsetAsync(ctr, 0, sizeof(uint32_t), s));

  Params p = make_params(ctx, opts, M);
  {
    // one chase launch serves every instance: its chains and block size come
    // from the class that holds most of the batch's elements
    const size_t k = std::max_element(class_elems.begin(), class_elems.end()) - class_elems.begin();
    if (!(opts && opts->chains_per_thread)) p.chains = ctx.class_chains[k];
    if (!(opts && opts->block_size)) p.block = (ctx.class_block[k] == 128 || ctx.class_block[k] == 512)
                                                   ? ctx.class_block[k] : 256u;
  }
  const uint32_t salt = mix32(p.seed ^ 0x62617463u);
  {
    ProfScope ps(ctx, "batch_prepare", s);
    const unsigned grid = (unsigned)std::min<uint64_t>(items.size(), (uint64_t)ctx.usable_sms() * 8);
    if (weights)
      k_batch_prepare<BWU32><<<grid, BP_THREADS, 0, s>>>(d_items, (uint32_t)items.size(), d_segs, in, BWU32{weights},
                                                         rec, fpar, ruler_elem, ctr, salt, ctx.d_status);
    else
      k_batch_prepare<BWUnit><<<grid, BP_THREADS, 0, s>>>(d_items, (uint32_t)items.size(), d_segs, in, BWUnit{}, rec,
                                                          fpar, ruler_elem, ctr, salt, ctx.d_status);
    KS_CHECK_LAUNCH();
  }
  KS_TRY(batch_tours(ctx, fpar, (uint32_t)F, d_fd, d_foff, d_fth, nf, (uint32_t)total, rec, ruler_elem, ctr,
                     mix32(p.seed ^ 0x70757254u), s));
  uint32_t r0 = 0;
  KS_TRY(read_u32(ctx, ctr, &r0, s));
  SinkBatch sink{root_out, rank_out, (uint32_t)total, reinterpret_cast<const uint64_t*>(d_off), d_hint, nseg};
  p.algorithm = KASCADE_ALGO_SPARSE_RULING_SET;
  return rank_records(ctx, rec, M, r0, ruler_elem, sink, p, s);
}

}  // namespace ks
