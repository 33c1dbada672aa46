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
//    both lanes' batches run concurrently on the device, and lane 1's
//    persistent kernels leave `latency_sms` SMs free for lane 0.
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
#include <thread>
#include <unordered_map>
#include <vector>

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

__global__ void k_fill_u32(uint32_t* __restrict__ p, uint64_t n, uint32_t v) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = v;
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
  uint32_t requests;
  uint64_t elements;
  double t_start, t_alloc, t_gathered, t_end;
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
  };
  Lane lanes[2];
  cudaStream_t copy_stream = nullptr;
  // batch buffers come from a pool that keeps freed memory (no release to
  // the driver, hence no device-wide synchronisation on reuse)
  cudaMemPool_t pool = nullptr;
  ResultHeap heap;

  std::vector<BatchTrace> trace;
  bool tracing = false;

  void admit_locked();
  void lane_loop(int lane);
  kascade_status warm_lane(int lane, uint64_t n_list, uint64_t n_forest);
};

// Run one synthetic batch (a list and a forest) on a lane before serving, so
// that the first requests pay for no kernel loading and no pool growth.
kascade_status kascade_server::warm_lane(int lane, uint64_t n_list, uint64_t n_forest) {
  Lane& L = lanes[lane];
  const uint64_t n = n_list + n_forest;
  if (n > L.cap || 16 * n > heap.size) return KASCADE_OK;  // nothing to warm with
  uint64_t* in = L.d_in;
  uint32_t* w = L.d_w;
  uint64_t* root = reinterpret_cast<uint64_t*>(heap.base);
  uint64_t* rank = root + n;
  kascade_status st = KASCADE_OK;
  if (st == KASCADE_OK) st = kascade_gen_list(n_list, 0x5e7e, 0, in, L.stream);
  if (st == KASCADE_OK) st = kascade_gen_weights(n, 0x5e7e, 16, w, L.stream);
  if (st == KASCADE_OK) st = kascade_gen_forest(n_forest, 0x5e7e, 0, 16, 0, in + n_list, L.stream);
  if (st == KASCADE_OK) {
    kascade_segment segs[2] = {{0, n_list, KASCADE_SEG_LIST, 0}, {n_list, n_forest, KASCADE_SEG_FOREST, 0}};
    kascade_opts o;
    kascade_opts_init(&o);
    st = kascade_rank_batch(L.ctx, segs, 2, in, w, n, root, rank, &o, L.stream);
  }
  if (cudaStreamSynchronize(L.stream) != cudaSuccess && st == KASCADE_OK) st = KASCADE_ERR_CUDA;
  cudaGetLastError();
  return st;
}

// Admit waiting requests while they fit the budget: arrival order, except
// that requests for the latency lane may pass larger ones that do not fit
// yet.  Admission is accounting only; the lane copies the input when it runs.
void kascade_server::admit_locked() {
  bool blocked_large = false;
  for (auto it = waiting.begin(); it != waiting.end();) {
    Request* r = *it;
    const bool small = r->n <= cfg.small_max;
    if (blocked_large && !small) {
      ++it;
      continue;
    }
    if (bytes_in_use + r->footprint > cfg.hbm_budget_bytes && bytes_in_use > 0) {
      if (!small) blocked_large = true;
      ++it;
      continue;
    }
    it = waiting.erase(it);
    bytes_in_use += r->footprint;
    r->admitted = true;
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
    cv_work.wait(lk, [&] {
      if (stop) return true;
      for (Request* r : ready)
        if (mine(r)) return true;
      return false;
    });
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
    const double t0 = now_s();
    auto b = std::make_shared<BatchBuf>();
    b->n = elems;
    b->heap_bytes = 16 * elems;
    b->heap_off = heap.alloc(b->heap_bytes);
    lk.unlock();
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
      if (cudaMallocFromPoolAsync(reinterpret_cast<void**>(&d_in), elems * 8, pool, L.stream) != cudaSuccess ||
          (any_w && cudaMallocFromPoolAsync(reinterpret_cast<void**>(&d_w), elems * 4, pool, L.stream) != cudaSuccess)) {
        cudaGetLastError();
        st = KASCADE_ERR_OOM;
      }
    }
    if (b->heap_off != NO_CHUNK) {
      b->d_root = reinterpret_cast<uint64_t*>(heap.base + b->heap_off);
      b->d_rank = b->d_root + elems;
    } else if (cudaMallocFromPoolAsync(reinterpret_cast<void**>(&b->d_root), elems * 16, pool, L.stream) ==
               cudaSuccess) {
      b->d_rank = b->d_root + elems;
    } else {
      cudaGetLastError();
      st = KASCADE_ERR_OOM;
    }
    const double t_alloc = now_s();
    std::vector<kascade_segment> segs(take.size());
    uint64_t off = 0;
    for (size_t i = 0; i < take.size() && st == KASCADE_OK; ++i) {
      Request* r = take[i];
      r->t_start = t0;
      segs[i] = kascade_segment{off, r->n, r->kind, 0};
      const void* in_src = r->src_in ? static_cast<const void*>(r->src_in) : static_cast<const void*>(r->h_in.data());
      const void* w_src = r->src_w ? static_cast<const void*>(r->src_w) : static_cast<const void*>(r->h_w.data());
      if (r->n) {
        if (cudaMemcpyAsync(d_in + off, in_src, r->n * 8, cudaMemcpyDefault, L.stream) != cudaSuccess)
          st = KASCADE_ERR_CUDA;
        if (any_w) {
          // lists without weights rank with unit weights; forests ignore weights
          cudaError_t e = cudaSuccess;
          if (r->has_w) {
            e = cudaMemcpyAsync(d_w + off, w_src, r->n * 4, cudaMemcpyDefault, L.stream);
          } else {
            k_fill_u32<<<(unsigned)std::min<uint64_t>((r->n + 255) / 256, 4096), 256, 0, L.stream>>>(
                d_w + off, r->n, r->kind == KASCADE_SEG_LIST ? 1u : 0u);
            e = cudaGetLastError();
          }
          if (e != cudaSuccess) st = KASCADE_ERR_CUDA;
        }
      }
      r->off = off;
      off += r->n;
    }
    const double t_gathered = now_s();
    if (st == KASCADE_OK) {
      kascade_opts o;
      kascade_opts_init(&o);
      st = kascade_rank_batch(L.ctx, segs.data(), (uint32_t)segs.size(), d_in, any_w ? d_w : nullptr, elems,
                              b->d_root, b->d_rank, &o, L.stream);
    }
    // the staged input is free for the next batch once the stream is done;
    // host submissions drop their copies then too
    if (!staged) {
      if (d_in) cudaFreeAsync(d_in, L.stream);
      if (d_w) cudaFreeAsync(d_w, L.stream);
    }
    cudaStreamSynchronize(L.stream);
    for (Request* r : take) {
      std::vector<uint64_t>().swap(r->h_in);
      std::vector<uint32_t>().swap(r->h_w);
    }
    const double t1 = now_s();
    lk.lock();
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
    if (tracing) trace.push_back(BatchTrace{lane, (uint32_t)take.size(), elems, t0, t_alloc, t_gathered, t1});
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
  c->max_batch_elements = 1ull << 26;
  c->small_max = 1ull << 20;
  c->small_batch_elements = 1ull << 23;
  c->latency_sms = 16;
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
  if (s->cfg.max_batch_elements == 0) s->cfg.max_batch_elements = 1ull << 26;
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
    if (keep > 0 && keep < sms) kascade_ctx_set_sm_budget(s->lanes[1].ctx, sms - keep);
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
      ok = kascade_ctx_reserve(L.ctx, kascade_scratch_bytes_root_forest(cap[i])) == KASCADE_OK &&
           cudaMalloc(reinterpret_cast<void**>(&L.d_in), cap[i] * 8) == cudaSuccess &&
           cudaMalloc(reinterpret_cast<void**>(&L.d_w), cap[i] * 4) == cudaSuccess;
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
  if (s->warm_lane(0, 1ull << 20, 1ull << 19) != KASCADE_OK || s->warm_lane(1, 1ull << 22, 1ull << 21) != KASCADE_OK) {
    kascade_server_destroy(s);
    return KASCADE_ERR_CUDA;
  }
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
    // one line per batch: lane, requests, elements, start, buffers
    // allocated, inputs issued, end (seconds on the steady clock)
    if (FILE* f = std::fopen(std::getenv("KASCADE_SERVER_TRACE"), "w")) {
      std::fprintf(f, "lane,requests,elements,t_start,t_alloc,t_gathered,t_end\n");
      for (const BatchTrace& b : s->trace)
        std::fprintf(f, "%d,%u,%llu,%.6f,%.6f,%.6f,%.6f\n", b.lane, b.requests, (unsigned long long)b.elements,
                     b.t_start, b.t_alloc, b.t_gathered, b.t_end);
      std::fclose(f);
    }
  }
  cudaSetDevice(s->cfg.device);
  cudaDeviceSynchronize();
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
  }
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
  s->t_first_submit = 0;
  s->t_last_done = 0;
  return KASCADE_OK;
}

}  // extern "C"
