// Serving: a request loop over the batched ranker.
//
//  - submit: a request (list ranking or tree rooting, host or device input)
//    is admitted when its HBM footprint fits the budget; admission copies its
//    input to the device, where input and result stay until released.
//    Requests that do not fit wait in arrival order and are admitted as
//    memory frees up.
//  - lanes: each lane is a worker thread with its own library context and
//    CUDA stream.  A lane takes every admitted request of its class that is
//    waiting when it becomes free (continuous batching), gathers their inputs
//    into one concatenated buffer and ranks them with one kascade_rank_batch
//    call.  Lane 0 serves requests up to `small_max` elements (the latency
//    lane, small batches, higher stream priority), lane 1 the larger ones;
//    both lanes' batches run concurrently on the device.
//  - results: each request's root and rank live in its batch's output
//    buffers until the request is released.
//  - stats: per-request latency (submit to completion), p50 / p99, throughput.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "ctx.cuh"

namespace {

using Clock = std::chrono::steady_clock;

double now_s() { return std::chrono::duration<double>(Clock::now().time_since_epoch()).count(); }

struct BatchBuf {
  uint64_t* d_in = nullptr;
  uint32_t* d_w = nullptr;
  uint64_t* d_root = nullptr;
  uint64_t* d_rank = nullptr;
  uint64_t n = 0;
  uint64_t bytes = 0;
  int refs = 0;
};

struct Request {
  uint64_t id = 0;
  uint32_t kind = 0;
  uint64_t n = 0;
  uint64_t* d_in = nullptr;  // owned until the request runs
  uint32_t* d_w = nullptr;
  std::vector<uint64_t> h_in;  // host submissions wait here until admitted
  std::vector<uint32_t> h_w;
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
  double t_first_submit = 0, t_last_done = 0;
  bool stop = false;
  struct Lane {
    kascade_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    std::thread th;
  };
  Lane lanes[2];
  cudaStream_t copy_stream = nullptr;

  void admit_locked();
  void lane_loop(int lane);
  kascade_status admit_one(Request* r);
};

// Copy a request's input to the device (caller holds no lock).
kascade_status kascade_server::admit_one(Request* r) {
  cudaSetDevice(cfg.device);
  const size_t in_bytes = r->n * sizeof(uint64_t), w_bytes = r->n * sizeof(uint32_t);
  if (cudaMallocAsync(reinterpret_cast<void**>(&r->d_in), in_bytes ? in_bytes : 8, copy_stream) != cudaSuccess)
    return cudaGetLastError(), KASCADE_ERR_OOM;
  if (r->has_w &&
      cudaMallocAsync(reinterpret_cast<void**>(&r->d_w), w_bytes ? w_bytes : 8, copy_stream) != cudaSuccess)
    return cudaGetLastError(), KASCADE_ERR_OOM;
  if (!r->h_in.empty()) {
    if (cudaMemcpyAsync(r->d_in, r->h_in.data(), in_bytes, cudaMemcpyHostToDevice, copy_stream) != cudaSuccess)
      return cudaGetLastError(), KASCADE_ERR_CUDA;
    if (r->has_w &&
        cudaMemcpyAsync(r->d_w, r->h_w.data(), w_bytes, cudaMemcpyHostToDevice, copy_stream) != cudaSuccess)
      return cudaGetLastError(), KASCADE_ERR_CUDA;
  }
  if (cudaStreamSynchronize(copy_stream) != cudaSuccess) return cudaGetLastError(), KASCADE_ERR_CUDA;
  std::vector<uint64_t>().swap(r->h_in);
  std::vector<uint32_t>().swap(r->h_w);
  return KASCADE_OK;
}

// Admit waiting host requests in arrival order while they fit the budget.
void kascade_server::admit_locked() {
  while (!waiting.empty()) {
    Request* r = waiting.front();
    if (bytes_in_use + r->footprint > cfg.hbm_budget_bytes && bytes_in_use > 0) break;
    waiting.pop_front();
    bytes_in_use += r->footprint;
    mu.unlock();
    kascade_status st = admit_one(r);
    mu.lock();
    if (st != KASCADE_OK) {
      r->state = 4;
      r->status = st;
      bytes_in_use -= r->footprint;
      cv_done.notify_all();
      continue;
    }
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
    lk.unlock();
    // gather into one concatenated batch and rank it
    const double t0 = now_s();
    auto b = std::make_shared<BatchBuf>();
    b->n = elems;
    bool any_w = false;
    for (Request* r : take) any_w |= r->has_w;
    kascade_status st = KASCADE_OK;
    if (cudaMallocAsync(reinterpret_cast<void**>(&b->d_in), elems * 8, L.stream) != cudaSuccess ||
        cudaMallocAsync(reinterpret_cast<void**>(&b->d_root), elems * 8, L.stream) != cudaSuccess ||
        cudaMallocAsync(reinterpret_cast<void**>(&b->d_rank), elems * 8, L.stream) != cudaSuccess ||
        (any_w && cudaMallocAsync(reinterpret_cast<void**>(&b->d_w), elems * 4, L.stream) != cudaSuccess)) {
      cudaGetLastError();
      st = KASCADE_ERR_OOM;
    }
    std::vector<kascade_segment> segs(take.size());
    uint64_t off = 0;
    for (size_t i = 0; i < take.size() && st == KASCADE_OK; ++i) {
      Request* r = take[i];
      r->t_start = t0;
      segs[i] = kascade_segment{off, r->n, r->kind, 0};
      if (r->n) {
        if (cudaMemcpyAsync(b->d_in + off, r->d_in, r->n * 8, cudaMemcpyDeviceToDevice, L.stream) != cudaSuccess)
          st = KASCADE_ERR_CUDA;
        if (any_w) {
          // lists without weights rank with unit weights; forests ignore weights
          cudaError_t e = cudaSuccess;
          if (r->has_w) {
            e = cudaMemcpyAsync(b->d_w + off, r->d_w, r->n * 4, cudaMemcpyDeviceToDevice, L.stream);
          } else {
            k_fill_u32<<<(unsigned)std::min<uint64_t>((r->n + 255) / 256, 4096), 256, 0, L.stream>>>(
                b->d_w + off, r->n, r->kind == KASCADE_SEG_LIST ? 1u : 0u);
            e = cudaGetLastError();
          }
          if (e != cudaSuccess) st = KASCADE_ERR_CUDA;
        }
      }
      r->off = off;
      off += r->n;
    }
    if (st == KASCADE_OK) {
      kascade_opts o;
      kascade_opts_init(&o);
      st = kascade_rank_batch(L.ctx, segs.data(), (uint32_t)segs.size(), b->d_in, any_w ? b->d_w : nullptr, elems,
                              b->d_root, b->d_rank, &o, L.stream);
    }
    // inputs are no longer needed: free them and the batch's concatenated input
    for (Request* r : take) {
      if (r->d_in) cudaFreeAsync(r->d_in, L.stream);
      if (r->d_w) cudaFreeAsync(r->d_w, L.stream);
      r->d_in = nullptr;
      r->d_w = nullptr;
    }
    if (b->d_in) cudaFreeAsync(b->d_in, L.stream);
    if (b->d_w) cudaFreeAsync(b->d_w, L.stream);
    b->d_in = nullptr;
    b->d_w = nullptr;
    cudaStreamSynchronize(L.stream);
    const double t1 = now_s();
    lk.lock();
    b->refs = (int)take.size();
    for (Request* r : take) {
      r->batch = b;
      r->t_done = t1;
      r->status = st;
      r->state = (st == KASCADE_OK) ? 3 : 4;
      // the input share of the footprint is released now; the result share
      // stays until the request is released
      const double lat = r->t_done - r->t_submit;
      latencies_all.push_back(lat);
      if (r->n <= cfg.small_max) latencies_small.push_back(lat);
      elements_done += r->n;
    }
    batches++;
    t_last_done = t1;
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
  c->max_batch_elements = 1ull << 28;
  c->small_max = 1ull << 20;
  c->small_batch_elements = 1ull << 23;
}

KASCADE_API kascade_status kascade_server_create(const kascade_server_config* cfg, kascade_server** out) {
  if (!out) return KASCADE_ERR_INVALID_ARG;
  *out = nullptr;
  auto* s = new (std::nothrow) kascade_server();
  if (!s) return KASCADE_ERR_OOM;
  kascade_server_config_init(&s->cfg);
  if (cfg) s->cfg = *cfg;
  if (s->cfg.max_batch_requests == 0) s->cfg.max_batch_requests = 4096;
  if (s->cfg.max_batch_elements == 0) s->cfg.max_batch_elements = 1ull << 28;
  if (s->cfg.hbm_budget_bytes == 0) s->cfg.hbm_budget_bytes = 40ull << 30;
  if (s->cfg.small_batch_elements == 0) s->cfg.small_batch_elements = 1ull << 23;
  if (cudaSetDevice(s->cfg.device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete s;
    return KASCADE_ERR_CUDA;
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
  cudaSetDevice(s->cfg.device);
  cudaDeviceSynchronize();
  for (auto& kv : s->reqs) {
    Request* r = kv.second.get();
    if (r->d_in) cudaFree(r->d_in);
    if (r->d_w) cudaFree(r->d_w);
  }
  std::vector<std::shared_ptr<BatchBuf>> bufs;
  for (auto& kv : s->reqs)
    if (kv.second->batch) bufs.push_back(kv.second->batch);
  s->reqs.clear();
  std::sort(bufs.begin(), bufs.end());
  bufs.erase(std::unique(bufs.begin(), bufs.end()), bufs.end());
  for (auto& b : bufs) {
    if (b->d_root) cudaFree(b->d_root);
    if (b->d_rank) cudaFree(b->d_rank);
    b->d_root = b->d_rank = nullptr;
  }
  for (auto& L : s->lanes) {
    if (L.ctx) kascade_ctx_destroy(L.ctx);
    if (L.stream) cudaStreamDestroy(L.stream);
  }
  if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
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
  std::unique_lock<std::mutex> lk(s->mu);
  if (r->footprint > s->cfg.hbm_budget_bytes) return KASCADE_ERR_TOO_LARGE;
  r->id = s->next_id++;
  *request_id = r->id;
  if (s->t_first_submit == 0) s->t_first_submit = r->t_submit;
  s->reqs.emplace(r->id, std::move(req));
  if (device) {
    // device input: copy into the server's own buffers at admission
    if (s->bytes_in_use + r->footprint > s->cfg.hbm_budget_bytes && s->bytes_in_use > 0) {
      // wait for memory: admission happens in order as requests are released
      s->cv_done.wait(lk, [&] { return s->bytes_in_use + r->footprint <= s->cfg.hbm_budget_bytes || s->bytes_in_use == 0; });
    }
    s->bytes_in_use += r->footprint;
    lk.unlock();
    cudaSetDevice(s->cfg.device);
    kascade_status st = KASCADE_OK;
    if (cudaMallocAsync(reinterpret_cast<void**>(&r->d_in), n ? n * 8 : 8, s->copy_stream) != cudaSuccess ||
        (n && cudaMemcpyAsync(r->d_in, input, n * 8, cudaMemcpyDeviceToDevice, s->copy_stream) != cudaSuccess))
      st = KASCADE_ERR_CUDA;
    if (st == KASCADE_OK && r->has_w &&
        (cudaMallocAsync(reinterpret_cast<void**>(&r->d_w), n ? n * 4 : 8, s->copy_stream) != cudaSuccess ||
         (n && cudaMemcpyAsync(r->d_w, weights, n * 4, cudaMemcpyDeviceToDevice, s->copy_stream) != cudaSuccess)))
      st = KASCADE_ERR_CUDA;
    if (cudaStreamSynchronize(s->copy_stream) != cudaSuccess) st = KASCADE_ERR_CUDA;
    lk.lock();
    if (st != KASCADE_OK) {
      cudaGetLastError();
      r->state = 4;
      r->status = st;
      s->bytes_in_use -= r->footprint;
      s->cv_done.notify_all();
      return st;
    }
    r->admitted = true;
    r->state = 1;
    s->ready.push_back(r);
    s->cv_work.notify_all();
    return KASCADE_OK;
  }
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
    if (r->batch && --r->batch->refs == 0) drop = r->batch;
    s->reqs.erase(it);
    s->admit_locked();
    s->cv_done.notify_all();
  }
  if (drop) {
    cudaSetDevice(s->cfg.device);
    if (drop->d_root) cudaFreeAsync(drop->d_root, s->copy_stream);
    if (drop->d_rank) cudaFreeAsync(drop->d_rank, s->copy_stream);
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
  return KASCADE_OK;
}

KASCADE_API kascade_status kascade_server_reset_stats(kascade_server* s) {
  if (!s) return KASCADE_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  s->latencies_all.clear();
  s->latencies_small.clear();
  s->elements_done = 0;
  s->batches = 0;
  s->t_first_submit = 0;
  s->t_last_done = 0;
  return KASCADE_OK;
}

}  // extern "C"
