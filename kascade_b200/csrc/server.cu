// Serving: a request loop over the batched ranker.
//
//  - submit: a request (list ranking or tree rooting, host or device input)
//    is admitted when its HBM footprint fits the budget.  Requests that do
//    not fit wait in arrival order and are admitted as memory frees up;
//    requests for the latency lane may pass larger ones that wait.  Host
//    inputs are held in host memory until their batch runs; the lane copies
//    every input of a batch straight into the batch's concatenated buffer.
//  - lanes: each lane is a worker thread with its own library context and
//    CUDA stream.  A lane takes every admitted request of its class that is
//    waiting when it becomes free (continuous batching), gathers their inputs
//    into one concatenated buffer and ranks them with one kascade_rank_batch
//    call.  Lane 0 serves requests up to `small_max` elements (the latency
//    lane, small batches, higher stream priority), lane 1 the larger ones;
//    both lanes' batches run concurrently on the device, and while lane 0
//    has work, lane 1's kernels are sized to leave `latency_sms` SMs free.
//    A batch's device-resident inputs are gathered by one kernel launch.
//  - memory: nothing is allocated per batch on the normal path.  Each lane
//    stages its batch input in buffers sized for a full batch, and results
//    go to a result heap set aside at creation (first fit, coalescing free
//    list kept on the host).  Only a request larger than a lane's batch limit,
//    or a batch that finds no room in the heap, allocates from the server's
//    memory pool (pool growth can stall the device for milliseconds).
//  - results: each request's root and rank live in its batch's output
//    buffers until the request is released.
//  - stats: per-request latency (submit to completion), p50 / p99, throughput.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda.h>

#include "ctx.cuh"

namespace {

using Clock = std::chrono::steady_clock;

double now_s() { return std::chrono::duration<double>(Clock::now().time_since_epoch()).count(); }

constexpr uint64_t NO_CHUNK = ~0ull;

struct BatchBuf {
  uint64_t* d_root = nullptr;  // results: root, then rank, in one chunk
  uint64_t* d_rank = nullptr;
  uint64_t n = 0;
  uint64_t heap_off = NO_CHUNK;  // offset in the result heap, or pool memory
  uint64_t heap_bytes = 0;
  int refs = 0;
};

// First-fit allocator over one device range, with coalescing on free.
struct ResultHeap {
  char* base = nullptr;
  uint64_t size = 0;
  std::map<uint64_t, uint64_t> free_blocks;  // offset -> bytes

  void init(char* p, uint64_t bytes) {
    base = p;
    size = bytes;
    free_blocks.clear();
    if (bytes) free_blocks.emplace(0, bytes);
  }
  uint64_t alloc(uint64_t bytes) {
    bytes = (bytes + 255) & ~255ull;
    for (auto it = free_blocks.begin(); it != free_blocks.end(); ++it) {
      if (it->second < bytes) continue;
      const uint64_t off = it->first, left = it->second - bytes;
      free_blocks.erase(it);
      if (left) free_blocks.emplace(off + bytes, left);
      return off;
    }
    return NO_CHUNK;
  }
  void release(uint64_t off, uint64_t bytes) {
    bytes = (bytes + 255) & ~255ull;
    auto it = free_blocks.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_blocks.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_blocks.erase(nx);
    }
    if (it != free_blocks.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_blocks.erase(it);
      }
    }
  }
};

struct Request {
  uint64_t id = 0;
  uint32_t kind = 0;
  uint64_t n = 0;
  std::vector<uint64_t> h_in;  // host submissions wait here until their batch runs
  std::vector<uint32_t> h_w;
  const uint64_t* src_in = nullptr;  // device submissions: copied from here when the batch runs
  const uint32_t* src_w = nullptr;
  uint64_t result_bytes = 0;  // the share of the footprint held until release
  bool has_w = false;
  bool admitted = false;
  int state = 0;  // 0 waiting for memory, 1 admitted, 2 running, 3 done, 4 failed
  kascade_status status = KASCADE_OK;
  std::shared_ptr<BatchBuf> batch;
  uint64_t off = 0;
  uint64_t footprint = 0;
  double t_submit = 0, t_start = 0, t_done = 0;
};

// One piece of a batch's input gather: up to PIECE elements of one request.
struct __align__(16) Piece {
  const uint64_t* src_in;  // nullptr: input already in place (host submission)
  const uint32_t* src_w;   // nullptr: fill the weights with `fill`
  uint64_t dst;            // offset in the batch
  uint32_t n;
  uint32_t fill;
};
constexpr uint32_t PIECE = 16384;
constexpr int LATENCY_HOLD_MS = 20;

// Gather device-resident request inputs (and weights, or their unit / zero
// fill) into the batch's concatenated buffers: one launch per batch.  A thread
// has GATHER_UNROLL independent loads in flight per round (one load at a time
// left the copy far below the HBM rate).
constexpr uint32_t GATHER_UNROLL = 4;
__global__ void __launch_bounds__(256) k_gather(const Piece* __restrict__ pieces, uint32_t npieces,
                                                uint64_t* __restrict__ d_in, uint32_t* __restrict__ d_w) {
  for (uint32_t p = blockIdx.x; p < npieces; p += gridDim.x) {
    const Piece pc = pieces[p];
    for (uint32_t i0 = threadIdx.x; i0 < pc.n; i0 += blockDim.x * GATHER_UNROLL) {
      unsigned long long v[GATHER_UNROLL];
      uint32_t wv[GATHER_UNROLL];
#pragma unroll
      for (uint32_t u = 0; u < GATHER_UNROLL; ++u) {
        const uint32_t i = i0 + u * blockDim.x;
        v[u] = 0;
        wv[u] = pc.fill;
        if (i < pc.n) {
          if (pc.src_in) v[u] = __ldcs(reinterpret_cast<const unsigned long long*>(pc.src_in) + i);
          if (d_w && pc.src_w) wv[u] = __ldcs(pc.src_w + i);
        }
      }
#pragma unroll
      for (uint32_t u = 0; u < GATHER_UNROLL; ++u) {
        const uint32_t i = i0 + u * blockDim.x;
        if (i >= pc.n) continue;
        if (pc.src_in) d_in[pc.dst + i] = v[u];
        if (d_w) d_w[pc.dst + i] = wv[u];
      }
    }
  }
}

uint64_t footprint_of(uint32_t kind, uint64_t n, bool w) {
  // input + weights + result (in its batch) + the batch's concatenated input
  // + ranking scratch (forests: sort, tour records and log on 2n tour slots)
  const uint64_t io = n * (8 + (w ? 4 : 0)) * 2 + 16 * n;
  const uint64_t scratch =
      kind == KASCADE_SEG_FOREST ? kascade_scratch_bytes_root_forest(n) : kascade_scratch_bytes_rank_list(n);
  return io + scratch - (192ull << 20);  // the fixed part of the scratch estimate is per lane, not per request
}

}  // namespace

// One finished batch, for the optional trace (KASCADE_SERVER_TRACE=<file>).
struct BatchTrace {
  int lane;
  int part;  // 1: ran in lane 1's SM partition
  uint32_t requests;
  uint64_t elements;
  double t_start, t_alloc, t_gathered, t_end;
  double gpu_ms, chase_ms;  // kernel time of the batch (trace runs profile it)
  char top[96];             // the batch's three longest kernels
};

struct kascade_server {
  kascade_server_config cfg{};
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> waiting;                       // not admitted (no memory yet)
  std::deque<Request*> ready;                         // admitted, not yet running
  std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
  std::vector<double> latencies_small, latencies_all;
  uint64_t next_id = 1;
  uint64_t bytes_in_use = 0;
  uint64_t elements_done = 0;
  uint64_t batches = 0;
  uint64_t lane_batches[2] = {0, 0}, lane_elements[2] = {0, 0};
  double lane_busy[2] = {0, 0}, lane_max[2] = {0, 0};
  double t_first_submit = 0, t_last_done = 0;
  bool stop = false;
  struct Lane {
    kascade_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    std::thread th;
    uint64_t* d_in = nullptr;  // staging for a full batch
    uint32_t* d_w = nullptr;
    uint64_t cap = 0;
    Piece* h_pieces = nullptr;  // gather table (pinned) and its device copy
    Piece* d_pieces = nullptr;
    uint64_t piece_cap = 0;
    // lane 1 only: a second context and stream inside the SM partition
    kascade_ctx* pctx = nullptr;
    cudaStream_t pstream = nullptr;
  };
  Lane lanes[2];
  cudaStream_t copy_stream = nullptr;
  // batch buffers come from a pool that keeps freed memory (no release to
  // the driver, hence no device-wide synchronisation on reuse)
  cudaMemPool_t pool = nullptr;
  ResultHeap heap;
  int lane1_busy_sms = 0;  // lane 1's SM budget while lane 0 has work (0 = all)
  // SM partition (green context) for lane 1 while lane 0 is active; lane 1
  // runs on the whole device otherwise
  CUgreenCtx green = nullptr;
  CUcontext green_cu = nullptr, primary_cu = nullptr;
  int partition_sms = 0;
  char* lane1_arena = nullptr;  // shared by lane 1's two contexts
  bool lane0_running = false;
  double lane0_last = -1e9;
  // continuous batching evidence: batches between take and completion, and
  // what was admitted or started while another batch was in flight
  int lanes_running = 0;
  uint64_t admitted_while_running = 0, batches_started_overlapping = 0;
  uint64_t partition_batches = 0;
  struct Driver {
    CUresult (*DeviceGet)(CUdevice*, int) = nullptr;
    CUresult (*DeviceGetDevResource)(CUdevice, CUdevResource*, CUdevResourceType) = nullptr;
    CUresult (*DevSmResourceSplitByCount)(CUdevResource*, unsigned int*, const CUdevResource*, CUdevResource*,
                                          unsigned int, unsigned int) = nullptr;
    CUresult (*DevResourceGenerateDesc)(CUdevResourceDesc*, CUdevResource*, unsigned int) = nullptr;
    CUresult (*GreenCtxCreate)(CUgreenCtx*, CUdevResourceDesc, CUdevice, unsigned int) = nullptr;
    CUresult (*GreenCtxDestroy)(CUgreenCtx) = nullptr;
    CUresult (*CtxFromGreenCtx)(CUcontext*, CUgreenCtx) = nullptr;
    CUresult (*CtxGetCurrent)(CUcontext*) = nullptr;
    CUresult (*CtxSetCurrent)(CUcontext) = nullptr;
  } drv;

  std::vector<BatchTrace> trace;
  bool tracing = false;

  void admit_locked();
  void lane_loop(int lane);
  kascade_status warm_lane(kascade_ctx* ctx, cudaStream_t stream, const Lane& L, uint64_t n_list, uint64_t n_forest);
  bool setup_partition();
  void drop_partition();
};

template <class F>
static bool driver_fn(const char* name, F*& fn) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q{};
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess ||
      !p) {
    cudaGetLastError();
    return false;
  }
  fn = reinterpret_cast<F*>(p);
  return true;
}

// Carve an SM partition of (all SMs - latency_sms, rounded down to the
// partition granularity of 8) as a green context, and give lane 1 a second
// library context and stream inside it.  Work in the partition cannot use
// the other SMs, so lane 0 always finds latency_sms SMs that lane 1 does not
// hold.  Returns false (and leaves lane 1 on the whole device, with grid
// budgets only) where the driver offers no green contexts.
bool kascade_server::setup_partition() {
  if (cfg.latency_sms == 0) return false;
  Driver& d = drv;
  if (!driver_fn("cuDeviceGet", d.DeviceGet) || !driver_fn("cuDeviceGetDevResource", d.DeviceGetDevResource) ||
      !driver_fn("cuDevSmResourceSplitByCount", d.DevSmResourceSplitByCount) ||
      !driver_fn("cuDevResourceGenerateDesc", d.DevResourceGenerateDesc) ||
      !driver_fn("cuGreenCtxCreate", d.GreenCtxCreate) || !driver_fn("cuGreenCtxDestroy", d.GreenCtxDestroy) ||
      !driver_fn("cuCtxFromGreenCtx", d.CtxFromGreenCtx) || !driver_fn("cuCtxGetCurrent", d.CtxGetCurrent) ||
      !driver_fn("cuCtxSetCurrent", d.CtxSetCurrent))
    return false;
  CUdevice dev = 0;
  if (d.DeviceGet(&dev, cfg.device) != CUDA_SUCCESS || d.CtxGetCurrent(&primary_cu) != CUDA_SUCCESS || !primary_cu)
    return false;
  CUdevResource all{}, grp{}, rest{};
  if (d.DeviceGetDevResource(dev, &all, CU_DEV_RESOURCE_TYPE_SM) != CUDA_SUCCESS) return false;
  const int want = ((int)all.sm.smCount - (int)cfg.latency_sms) & ~7;
  if (want < 8) return false;
  unsigned int nb = 1;
  CUdevResourceDesc desc = nullptr;
  if (d.DevSmResourceSplitByCount(&grp, &nb, &all, &rest, 0, (unsigned)want) != CUDA_SUCCESS || nb < 1 ||
      d.DevResourceGenerateDesc(&desc, &grp, 1) != CUDA_SUCCESS ||
      d.GreenCtxCreate(&green, desc, dev, CU_GREEN_CTX_DEFAULT_STREAM) != CUDA_SUCCESS)
    return false;
  partition_sms = (int)grp.sm.smCount;
  Lane& L = lanes[1];
  bool ok = d.CtxFromGreenCtx(&green_cu, green) == CUDA_SUCCESS && d.CtxSetCurrent(green_cu) == CUDA_SUCCESS;
  if (ok) {
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    ok = cudaStreamCreateWithPriority(&L.pstream, cudaStreamNonBlocking, lo) == cudaSuccess &&
         kascade_ctx_create(cfg.device, &L.pctx) == KASCADE_OK;
  }
  if (ok) {
    kascade_ctx_set_sm_budget(L.pctx, partition_sms);
    ks::arena_adopt(*L.pctx, lane1_arena, kascade_scratch_bytes_root_forest(L.cap));
    ok = warm_lane(L.pctx, L.pstream, L, 1ull << 22, 1ull << 21) == KASCADE_OK;
  }
  d.CtxSetCurrent(primary_cu);
  cudaGetLastError();
  if (!ok) drop_partition();
  return ok;
}

void kascade_server::drop_partition() {
  Lane& L = lanes[1];
  if (green_cu && drv.CtxSetCurrent) {
    drv.CtxSetCurrent(green_cu);
    if (L.pctx) kascade_ctx_destroy(L.pctx);
    if (L.pstream) cudaStreamDestroy(L.pstream);
    drv.CtxSetCurrent(primary_cu);
  }
  L.pctx = nullptr;
  L.pstream = nullptr;
  if (green && drv.GreenCtxDestroy) drv.GreenCtxDestroy(green);
  green = nullptr;
  green_cu = nullptr;
  partition_sms = 0;
  cudaGetLastError();
}

// Run one synthetic batch (a list and a forest) on a lane before serving, so
// that the first requests pay for no kernel loading and no pool growth.
kascade_status kascade_server::warm_lane(kascade_ctx* ctx, cudaStream_t stream, const Lane& L, uint64_t n_list,
                                         uint64_t n_forest) {
  const uint64_t n = n_list + n_forest;
  if (n > L.cap || 16 * n > heap.size) return KASCADE_OK;  // nothing to warm with
  uint64_t* in = L.d_in;
  uint32_t* w = L.d_w;
  uint64_t* root = reinterpret_cast<uint64_t*>(heap.base);
  uint64_t* rank = root + n;
  kascade_status st = KASCADE_OK;
  if (st == KASCADE_OK) st = kascade_gen_list(n_list, 0x5e7e, 0, in, stream);
  if (st == KASCADE_OK) st = kascade_gen_weights(n, 0x5e7e, 16, w, stream);
  if (st == KASCADE_OK) st = kascade_gen_forest(n_forest, 0x5e7e, 0, 16, 0, in + n_list, stream);
  if (st == KASCADE_OK) {
    // an empty gather, to load the gather kernel in this context too
    k_gather<<<1, 256, 0, stream>>>(L.d_pieces, 0, in, w);
    if (cudaGetLastError() != cudaSuccess) st = KASCADE_ERR_CUDA;
  }
  if (st == KASCADE_OK) {
    kascade_segment segs[2] = {{0, n_list, KASCADE_SEG_LIST, 0}, {n_list, n_forest, KASCADE_SEG_FOREST, 0}};
    kascade_opts o;
    kascade_opts_init(&o);
    st = kascade_rank_batch(ctx, segs, 2, in, w, n, root, rank, &o, stream);
  }
  if (cudaStreamSynchronize(stream) != cudaSuccess && st == KASCADE_OK) st = KASCADE_ERR_CUDA;
  cudaGetLastError();
  return st;
}

// Admit waiting requests while they fit the budget: arrival order, except
// that requests for the latency lane may pass larger ones that do not fit
// yet.  Admission is accounting only; the lane copies the input when it runs.
void kascade_server::admit_locked() {
  bool blocked_large = false;
  // large requests stop short of the share kept for the latency lane
  const uint64_t reserve = cfg.hbm_budget_bytes / 100 * std::min<uint32_t>(cfg.small_reserve_pct, 90);
  for (auto it = waiting.begin(); it != waiting.end();) {
    Request* r = *it;
    const bool small = r->n <= cfg.small_max;
    if (blocked_large && !small) {
      ++it;
      continue;
    }
    const uint64_t limit = small ? cfg.hbm_budget_bytes : cfg.hbm_budget_bytes - reserve;
    if (bytes_in_use + r->footprint > limit && bytes_in_use > 0) {
      if (!small) blocked_large = true;
      ++it;
      continue;
    }
    it = waiting.erase(it);
    bytes_in_use += r->footprint;
    r->admitted = true;
    if (lanes_running > 0) admitted_while_running++;
    r->state = 1;
    ready.push_back(r);
    cv_work.notify_all();
  }
}

void kascade_server::lane_loop(int lane) {
  Lane& L = lanes[lane];
  cudaSetDevice(cfg.device);
  std::unique_lock<std::mutex> lk(mu);
  while (true) {
    // take every ready request of this lane's class (up to the batch limits)
    std::vector<Request*> take;
    uint64_t elems = 0;
    auto mine = [&](const Request* r) { return lane == 0 ? r->n <= cfg.small_max : r->n > cfg.small_max; };
    const uint64_t max_elems = lane == 0 ? cfg.small_batch_elements : cfg.max_batch_elements;
    auto have_work = [&] {
      for (Request* r : ready)
        if (mine(r)) return true;
      return false;
    };
    if (lane == 0 && !have_work() && !stop) {
      // give lane 1 all SMs back only after the latency lane has been idle
      // for a while: arrivals are bursty, and a full-width launch of lane 1
      // holds its SMs until it ends
      if (!cv_work.wait_for(lk, std::chrono::milliseconds(LATENCY_HOLD_MS), [&] { return stop || have_work(); }))
        kascade_ctx_set_sm_budget(lanes[1].ctx, 0);
    }
    cv_work.wait(lk, [&] { return stop || have_work(); });
    if (stop && ready.empty()) break;
    for (auto it = ready.begin(); it != ready.end();) {
      Request* r = *it;
      if (mine(r) && take.size() < cfg.max_batch_requests && (take.empty() || elems + r->n <= max_elems)) {
        take.push_back(r);
        elems += r->n;
        r->state = 2;
        it = ready.erase(it);
      } else {
        ++it;
      }
    }
    if (take.empty()) {
      if (stop) break;
      continue;
    }
    if (lanes_running > 0) batches_started_overlapping++;
    lanes_running++;
    // while the latency lane has work, the throughput lane's next launches
    // leave it latency_sms SMs, and its next batch runs in the partition
    const double t0 = now_s();
    if (lane == 0) {
      kascade_ctx_set_sm_budget(lanes[1].ctx, lane1_busy_sms);
      lane0_running = true;
    }
    bool in_part = false;
    if (lane == 1 && L.pctx) {
      bool small_waiting = false;
      for (Request* r : ready) small_waiting |= r->n <= cfg.small_max;
      in_part = lane0_running || small_waiting || t0 - lane0_last < 1e-3 * LATENCY_HOLD_MS;
      if (in_part) partition_batches++;
    }
    kascade_ctx* C = in_part ? L.pctx : L.ctx;
    cudaStream_t S = in_part ? L.pstream : L.stream;
    auto b = std::make_shared<BatchBuf>();
    b->n = elems;
    b->heap_bytes = 16 * elems;
    b->heap_off = heap.alloc(b->heap_bytes);
    lk.unlock();
    if (lane == 1 && green_cu) drv.CtxSetCurrent(in_part ? green_cu : primary_cu);
    // gather into one concatenated batch and rank it
    bool any_w = false;
    for (Request* r : take) any_w |= r->has_w;
    kascade_status st = KASCADE_OK;
    uint64_t* d_in = L.d_in;
    uint32_t* d_w = L.d_w;
    const bool staged = elems <= L.cap;
    if (!staged) {
      d_in = nullptr;
      d_w = nullptr;
      if (cudaMallocFromPoolAsync(reinterpret_cast<void**>(&d_in), elems * 8, pool, S) != cudaSuccess ||
          (any_w && cudaMallocFromPoolAsync(reinterpret_cast<void**>(&d_w), elems * 4, pool, S) != cudaSuccess)) {
        cudaGetLastError();
        st = KASCADE_ERR_OOM;
      }
    }
    if (b->heap_off != NO_CHUNK) {
      b->d_root = reinterpret_cast<uint64_t*>(heap.base + b->heap_off);
      b->d_rank = b->d_root + elems;
    } else if (cudaMallocFromPoolAsync(reinterpret_cast<void**>(&b->d_root), elems * 16, pool, S) ==
               cudaSuccess) {
      b->d_rank = b->d_root + elems;
    } else {
      cudaGetLastError();
      st = KASCADE_ERR_OOM;
    }
    const double t_alloc = now_s();
    std::vector<kascade_segment> segs(take.size());
    uint64_t off = 0;
    uint64_t np = 0;
    std::vector<Piece> big;  // table overflow (a request beyond the lane's batch limit)
    auto add_piece = [&](const Piece& pc) {
      if (np < L.piece_cap) L.h_pieces[np] = pc;
      else big.push_back(pc);
      ++np;
    };
    for (size_t i = 0; i < take.size() && st == KASCADE_OK; ++i) {
      Request* r = take[i];
      r->t_start = t0;
      segs[i] = kascade_segment{off, r->n, r->kind, 0};
      // lists without weights rank with unit weights; forests ignore weights
      const uint32_t fill = r->kind == KASCADE_SEG_LIST ? 1u : 0u;
      if (r->n && !r->src_in) {
        // host submission: copy now, the gather kernel fills missing weights
        if (cudaMemcpyAsync(d_in + off, r->h_in.data(), r->n * 8, cudaMemcpyHostToDevice, S) != cudaSuccess ||
            (any_w && r->has_w &&
             cudaMemcpyAsync(d_w + off, r->h_w.data(), r->n * 4, cudaMemcpyHostToDevice, S) != cudaSuccess))
          st = KASCADE_ERR_CUDA;
        if (any_w && !r->has_w)
          for (uint64_t k = 0; k < r->n; k += PIECE)
            add_piece(Piece{nullptr, nullptr, off + k, (uint32_t)std::min<uint64_t>(PIECE, r->n - k), fill});
      } else {
        for (uint64_t k = 0; k < r->n; k += PIECE)
          add_piece(Piece{r->src_in + k, r->src_w ? r->src_w + k : nullptr, off + k,
                          (uint32_t)std::min<uint64_t>(PIECE, r->n - k), fill});
      }
      r->off = off;
      off += r->n;
    }
    if (st == KASCADE_OK && np) {
      Piece* table = L.d_pieces;
      bool own_table = false;
      if (!big.empty()) {
        // rare: a table larger than the lane's; copy it whole from pageable memory
        std::vector<Piece> all(L.h_pieces, L.h_pieces + L.piece_cap);
        all.insert(all.end(), big.begin(), big.end());
        table = nullptr;
        own_table = true;
        if (cudaMallocFromPoolAsync(reinterpret_cast<void**>(&table), np * sizeof(Piece), pool, S) !=
                cudaSuccess ||
            cudaMemcpyAsync(table, all.data(), np * sizeof(Piece), cudaMemcpyHostToDevice, S) != cudaSuccess)
          st = KASCADE_ERR_CUDA;
      } else if (cudaMemcpyAsync(table, L.h_pieces, np * sizeof(Piece), cudaMemcpyHostToDevice, S) !=
                 cudaSuccess) {
        st = KASCADE_ERR_CUDA;
      }
      if (st == KASCADE_OK) {
        const unsigned grid = (unsigned)std::min<uint64_t>(np, 148ull * 8);
        k_gather<<<grid, 256, 0, S>>>(table, (uint32_t)np, d_in, any_w ? d_w : nullptr);
        if (cudaGetLastError() != cudaSuccess) st = KASCADE_ERR_CUDA;
      }
      if (own_table && table) cudaFreeAsync(table, S);
      cudaGetLastError();
    }
    const double t_gathered = now_s();
    if (st == KASCADE_OK) {
      kascade_opts o;
      kascade_opts_init(&o);
      o.profile = tracing ? 1 : 0;
      // Both lanes enqueue their whole recursion at once (one host wait per
      // batch).  The throughput lane took the host-driven recursion before,
      // so that each level's launches took the SM budget in force when made;
      // with its batches in the SM partition while the latency lane has work,
      // the device-driven form serves 3% more (1.16 -> 1.19e10 elements/s on
      // the 20k req/s mix) for 0.4 ms more on the <=2^20 p99 (3.9 -> 4.3 ms).
      st = kascade_rank_batch(C, segs.data(), (uint32_t)segs.size(), d_in, any_w ? d_w : nullptr, elems, b->d_root,
                              b->d_rank, &o, S);
    }
    // the staged input is free for the next batch once the stream is done;
    // host submissions drop their copies then too
    if (!staged) {
      if (d_in) cudaFreeAsync(d_in, S);
      if (d_w) cudaFreeAsync(d_w, S);
    }
    cudaStreamSynchronize(S);
    for (Request* r : take) {
      std::vector<uint64_t>().swap(r->h_in);
      std::vector<uint32_t>().swap(r->h_w);
    }
    const double t1 = now_s();
    lk.lock();
    lanes_running--;
    if (lane == 0) {
      lane0_running = false;
      lane0_last = t1;
    }
    b->refs = (int)take.size();
    for (Request* r : take) {
      r->batch = b;
      r->t_done = t1;
      r->status = st;
      r->state = (st == KASCADE_OK) ? 3 : 4;
      // input and scratch shares of the footprint return to the budget now;
      // the result share stays until the request is released
      bytes_in_use -= (r->footprint - r->result_bytes);
      r->footprint = r->result_bytes;
      const double lat = r->t_done - r->t_submit;
      latencies_all.push_back(lat);
      if (r->n <= cfg.small_max) latencies_small.push_back(lat);
      elements_done += r->n;
    }
    batches++;
    lane_batches[lane]++;
    lane_elements[lane] += elems;
    lane_busy[lane] += t1 - t0;
    lane_max[lane] = std::max(lane_max[lane], t1 - t0);
    if (tracing) {
      double gpu = 0, chase = 0;
      std::vector<std::pair<double, std::string>> ks;
      for (auto& kv : C->times) {
        gpu += kv.second.first;
        if (kv.first == "chase") chase += kv.second.first;
        ks.emplace_back(kv.second.first, kv.first);
      }
      C->times.clear();
      std::sort(ks.rbegin(), ks.rend());
      BatchTrace bt{lane, in_part ? 1 : 0, (uint32_t)take.size(), elems, t0, t_alloc, t_gathered, t1, gpu, chase, {0}};
      std::string top;
      for (size_t i = 0; i < ks.size() && i < 3; ++i) {
        char buf[48];
        std::snprintf(buf, sizeof(buf), "%s%s=%.2f", i ? " " : "", ks[i].second.c_str(), ks[i].first);
        top += buf;
      }
      std::snprintf(bt.top, sizeof(bt.top), "%s", top.c_str());
      trace.push_back(bt);
    }
    t_last_done = t1;
    admit_locked();
    cv_done.notify_all();
  }
}

extern "C" {

KASCADE_API void kascade_server_config_init(kascade_server_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->struct_size = sizeof(kascade_server_config);
  c->device = 0;
  c->hbm_budget_bytes = 40ull << 30;
  c->max_batch_requests = 4096;
  c->max_batch_elements = 1ull << 27;
  c->small_max = 1ull << 20;
  c->small_batch_elements = 1ull << 23;
  c->latency_sms = 32;
  c->small_reserve_pct = 10;
  c->result_heap_bytes = 0;
}

KASCADE_API kascade_status kascade_server_create(const kascade_server_config* cfg, kascade_server** out) {
  if (!out) return KASCADE_ERR_INVALID_ARG;
  *out = nullptr;
  auto* s = new (std::nothrow) kascade_server();
  if (!s) return KASCADE_ERR_OOM;
  kascade_server_config_init(&s->cfg);
  if (cfg) s->cfg = *cfg;
  if (s->cfg.max_batch_requests == 0) s->cfg.max_batch_requests = 4096;
  if (s->cfg.max_batch_elements == 0) s->cfg.max_batch_elements = 1ull << 27;
  if (s->cfg.hbm_budget_bytes == 0) s->cfg.hbm_budget_bytes = 40ull << 30;
  if (s->cfg.small_batch_elements == 0) s->cfg.small_batch_elements = 1ull << 23;
  if (cudaSetDevice(s->cfg.device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete s;
    return KASCADE_ERR_CUDA;
  }
  {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = s->cfg.device;
    uint64_t keep_all = ~0ull;
    if (cudaMemPoolCreate(&s->pool, &props) != cudaSuccess ||
        cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep_all) != cudaSuccess) {
      cudaGetLastError();
      kascade_server_destroy(s);
      return KASCADE_ERR_CUDA;
    }
  }
  for (int i = 0; i < 2; ++i) {
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    // the latency lane gets the higher stream priority
    if (cudaStreamCreateWithPriority(&s->lanes[i].stream, cudaStreamNonBlocking, i == 0 ? hi : lo) != cudaSuccess ||
        kascade_ctx_create(s->cfg.device, &s->lanes[i].ctx) != KASCADE_OK) {
      cudaGetLastError();
      kascade_server_destroy(s);
      return KASCADE_ERR_CUDA;
    }
  }
  {
    // the throughput lane's persistent kernels leave SMs to the latency lane
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->cfg.device);
    const int keep = (int)s->cfg.latency_sms;
    if (keep > 0 && keep < sms) s->lane1_busy_sms = sms - keep;
  }
  // scratch and input staging for a full batch of each lane, so that no
  // batch grows an arena (growing synchronises the device and would stall
  // the other lane), and the result heap
  {
    const uint64_t cap[2] = {s->cfg.small_batch_elements, s->cfg.max_batch_elements};
    bool ok = true;
    for (int i = 0; i < 2 && ok; ++i) {
      kascade_server::Lane& L = s->lanes[i];
      L.cap = cap[i];
      L.piece_cap = cap[i] / PIECE + s->cfg.max_batch_requests + 1;
      const uint64_t scratch = kascade_scratch_bytes_root_forest(cap[i]);
      if (i == 1) {
        ok = cudaMalloc(reinterpret_cast<void**>(&s->lane1_arena), scratch) == cudaSuccess;
        if (ok) ks::arena_adopt(*L.ctx, s->lane1_arena, scratch);
      } else {
        ok = kascade_ctx_reserve(L.ctx, scratch) == KASCADE_OK;
      }
      ok = ok && cudaMalloc(reinterpret_cast<void**>(&L.d_in), cap[i] * 8) == cudaSuccess &&
           cudaMalloc(reinterpret_cast<void**>(&L.d_w), cap[i] * 4) == cudaSuccess &&
           cudaMallocHost(reinterpret_cast<void**>(&L.h_pieces), L.piece_cap * sizeof(Piece)) == cudaSuccess &&
           cudaMalloc(reinterpret_cast<void**>(&L.d_pieces), L.piece_cap * sizeof(Piece)) == cudaSuccess;
    }
    uint64_t hb = s->cfg.result_heap_bytes ? s->cfg.result_heap_bytes : s->cfg.hbm_budget_bytes / 2;
    hb = (hb + 255) & ~255ull;
    char* hp = nullptr;
    ok = ok && cudaMalloc(reinterpret_cast<void**>(&hp), hb) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      if (hp) cudaFree(hp);
      kascade_server_destroy(s);
      return KASCADE_ERR_OOM;
    }
    s->heap.init(hp, hb);
  }
  if (s->warm_lane(s->lanes[0].ctx, s->lanes[0].stream, s->lanes[0], 1ull << 20, 1ull << 19) != KASCADE_OK ||
      s->warm_lane(s->lanes[1].ctx, s->lanes[1].stream, s->lanes[1], 1ull << 22, 1ull << 21) != KASCADE_OK) {
    kascade_server_destroy(s);
    return KASCADE_ERR_CUDA;
  }
  s->setup_partition();
  s->tracing = std::getenv("KASCADE_SERVER_TRACE") != nullptr;
  for (int i = 0; i < 2; ++i) s->lanes[i].th = std::thread([s, i] { s->lane_loop(i); });
  *out = s;
  return KASCADE_OK;
}

KASCADE_API kascade_status kascade_server_destroy(kascade_server* s) {
  if (!s) return KASCADE_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv_work.notify_all();
  }
  for (auto& L : s->lanes)
    if (L.th.joinable()) L.th.join();
  if (s->tracing) {
    // one line per batch: lane, in the partition, requests, elements, start, buffers
    // allocated, inputs issued, end (seconds on the steady clock), summed
    // kernel time and chase kernel time (ms), the three longest kernels
    if (FILE* f = std::fopen(std::getenv("KASCADE_SERVER_TRACE"), "w")) {
      std::fprintf(f, "lane,part,requests,elements,t_start,t_alloc,t_gathered,t_end,gpu_ms,chase_ms,top\n");
      for (const BatchTrace& b : s->trace)
        std::fprintf(f, "%d,%d,%u,%llu,%.6f,%.6f,%.6f,%.6f,%.4f,%.4f,%s\n", b.lane, b.part, b.requests,
                     (unsigned long long)b.elements, b.t_start, b.t_alloc, b.t_gathered, b.t_end, b.gpu_ms, b.chase_ms,
                     b.top);
      std::fclose(f);
    }
  }
  cudaSetDevice(s->cfg.device);
  cudaDeviceSynchronize();
  s->drop_partition();
  std::vector<std::shared_ptr<BatchBuf>> bufs;
  for (auto& kv : s->reqs)
    if (kv.second->batch) bufs.push_back(kv.second->batch);
  s->reqs.clear();
  std::sort(bufs.begin(), bufs.end());
  bufs.erase(std::unique(bufs.begin(), bufs.end()), bufs.end());
  for (auto& b : bufs) {
    if (b->heap_off == NO_CHUNK && b->d_root) cudaFree(b->d_root);
    b->d_root = b->d_rank = nullptr;
  }
  if (s->heap.base) cudaFree(s->heap.base);
  for (auto& L : s->lanes) {
    if (L.ctx) kascade_ctx_destroy(L.ctx);
    if (L.stream) cudaStreamDestroy(L.stream);
    if (L.d_in) cudaFree(L.d_in);
    if (L.d_w) cudaFree(L.d_w);
    if (L.h_pieces) cudaFreeHost(L.h_pieces);
    if (L.d_pieces) cudaFree(L.d_pieces);
  }
  if (s->lane1_arena) cudaFree(s->lane1_arena);
  if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
  if (s->pool) cudaMemPoolDestroy(s->pool);
  cudaGetLastError();
  delete s;
  return KASCADE_OK;
}

static kascade_status submit(kascade_server* s, uint32_t kind, const uint64_t* input, const uint32_t* weights,
                             uint64_t n, bool device, uint64_t* request_id) {
  if (!s || !request_id || (n && !input) || (kind != KASCADE_SEG_LIST && kind != KASCADE_SEG_FOREST) ||
      n > 0x7FFFFFFFull)
    return KASCADE_ERR_INVALID_ARG;
  auto req = std::make_unique<Request>();
  Request* r = req.get();
  r->kind = kind;
  r->n = n;
  r->has_w = weights != nullptr && kind == KASCADE_SEG_LIST;
  r->footprint = footprint_of(kind, n, r->has_w);
  r->t_submit = now_s();
  if (!device) {
    r->h_in.assign(input, input + n);
    if (r->has_w) r->h_w.assign(weights, weights + n);
  }
  if (device) {
    r->src_in = input;
    r->src_w = r->has_w ? weights : nullptr;
  }
  r->result_bytes = 16 * n;
  std::unique_lock<std::mutex> lk(s->mu);
  if (r->footprint > s->cfg.hbm_budget_bytes) return KASCADE_ERR_TOO_LARGE;
  r->id = s->next_id++;
  *request_id = r->id;
  if (s->t_first_submit == 0) s->t_first_submit = r->t_submit;
  s->reqs.emplace(r->id, std::move(req));
  s->waiting.push_back(r);
  s->admit_locked();
  return KASCADE_OK;
}

KASCADE_API kascade_status kascade_server_submit(kascade_server* s, uint32_t kind, const uint64_t* input,
                                                 const uint32_t* weights, uint64_t n, uint64_t* request_id) {
  return submit(s, kind, input, weights, n, false, request_id);
}

KASCADE_API kascade_status kascade_server_submit_device(kascade_server* s, uint32_t kind, const uint64_t* input,
                                                        const uint32_t* weights, uint64_t n, uint64_t* request_id) {
  return submit(s, kind, input, weights, n, true, request_id);
}

KASCADE_API kascade_status kascade_server_wait(kascade_server* s, uint64_t id, double timeout_s) {
  if (!s) return KASCADE_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return KASCADE_ERR_INVALID_ARG;
  Request* r = it->second.get();
  auto done = [&] { return r->state >= 3; };
  if (timeout_s < 0) {
    s->cv_done.wait(lk, done);
  } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done)) {
    return KASCADE_ERR_TIMEOUT;
  }
  return r->status;
}

KASCADE_API kascade_status kascade_server_result_device(kascade_server* s, uint64_t id, const uint64_t** root,
                                                        const uint64_t** rank) {
  if (!s || !root || !rank) return KASCADE_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end() || it->second->state != 3) return KASCADE_ERR_INVALID_ARG;
  Request* r = it->second.get();
  *root = r->batch->d_root + r->off;
  *rank = r->batch->d_rank + r->off;
  return KASCADE_OK;
}

KASCADE_API kascade_status kascade_server_fetch(kascade_server* s, uint64_t id, uint64_t* root_out,
                                                uint64_t* rank_out) {
  const uint64_t *dr = nullptr, *dk = nullptr;
  kascade_status st = kascade_server_result_device(s, id, &dr, &dk);
  if (st != KASCADE_OK) return st;
  uint64_t n = 0;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    n = s->reqs[id]->n;
  }
  cudaSetDevice(s->cfg.device);
  if ((n && cudaMemcpyAsync(root_out, dr, n * 8, cudaMemcpyDeviceToHost, s->copy_stream) != cudaSuccess) ||
      (n && cudaMemcpyAsync(rank_out, dk, n * 8, cudaMemcpyDeviceToHost, s->copy_stream) != cudaSuccess) ||
      cudaStreamSynchronize(s->copy_stream) != cudaSuccess) {
    cudaGetLastError();
    return KASCADE_ERR_CUDA;
  }
  return KASCADE_OK;
}

KASCADE_API kascade_status kascade_server_release(kascade_server* s, uint64_t id) {
  if (!s) return KASCADE_ERR_INVALID_ARG;
  std::shared_ptr<BatchBuf> drop;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end() || it->second->state < 3) return KASCADE_ERR_INVALID_ARG;
    Request* r = it->second.get();
    s->bytes_in_use -= r->footprint;
    if (r->batch && --r->batch->refs == 0) {
      if (r->batch->heap_off != NO_CHUNK) {
        s->heap.release(r->batch->heap_off, r->batch->heap_bytes);
        r->batch->d_root = r->batch->d_rank = nullptr;
      } else {
        drop = r->batch;
      }
    }
    s->reqs.erase(it);
    s->admit_locked();
    s->cv_done.notify_all();
  }
  if (drop) {
    cudaSetDevice(s->cfg.device);
    if (drop->d_root) cudaFreeAsync(drop->d_root, s->copy_stream);
    drop->d_root = drop->d_rank = nullptr;
  }
  return KASCADE_OK;
}

static double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = q * (double)(v.size() - 1);
  const size_t lo = (size_t)pos;
  const size_t hi = std::min(lo + 1, v.size() - 1);
  return v[lo] + (v[hi] - v[lo]) * (pos - (double)lo);
}

KASCADE_API kascade_status kascade_server_get_stats(kascade_server* s, kascade_server_stats* out) {
  if (!s || !out) return KASCADE_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(out, 0, sizeof(*out));
  out->completed = s->latencies_all.size();
  out->batches = s->batches;
  out->elements = s->elements_done;
  out->p50_ms = 1e3 * percentile(s->latencies_all, 0.50);
  out->p99_ms = 1e3 * percentile(s->latencies_all, 0.99);
  out->p50_small_ms = 1e3 * percentile(s->latencies_small, 0.50);
  out->p99_small_ms = 1e3 * percentile(s->latencies_small, 0.99);
  out->completed_small = s->latencies_small.size();
  const double span = s->t_last_done - s->t_first_submit;
  out->elements_per_s = span > 0 ? (double)s->elements_done / span : 0.0;
  out->requests_per_s = span > 0 ? (double)s->latencies_all.size() / span : 0.0;
  out->bytes_in_use = s->bytes_in_use;
  for (int i = 0; i < 2; ++i) {
    out->lane_batches[i] = s->lane_batches[i];
    out->lane_elements[i] = s->lane_elements[i];
    out->lane_busy_ms[i] = 1e3 * s->lane_busy[i];
    out->lane_max_batch_ms[i] = 1e3 * s->lane_max[i];
  }
  out->partition_sms = (uint64_t)s->partition_sms;
  out->partition_batches = s->partition_batches;
  out->admitted_while_running = s->admitted_while_running;
  out->batches_started_overlapping = s->batches_started_overlapping;
  return KASCADE_OK;
}

KASCADE_API kascade_status kascade_server_reset_stats(kascade_server* s) {
  if (!s) return KASCADE_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  s->latencies_all.clear();
  s->latencies_small.clear();
  s->elements_done = 0;
  s->batches = 0;
  for (int i = 0; i < 2; ++i) {
    s->lane_batches[i] = s->lane_elements[i] = 0;
    s->lane_busy[i] = s->lane_max[i] = 0;
  }
  s->partition_batches = 0;
  s->admitted_while_running = 0;
  s->batches_started_overlapping = 0;
  s->t_first_submit = 0;
  s->t_last_done = 0;
  return KASCADE_OK;
}

}  // extern "C"
