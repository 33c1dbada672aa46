// Context plumbing: arena, status word, read-backs, kernel timing.
#include "ctx.cuh"

namespace ks {

kascade_status cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return KASCADE_OK;
  if (e == cudaErrorMemoryAllocation) return KASCADE_ERR_OOM;
  return KASCADE_ERR_CUDA;
}

kascade_status arena_begin_call(kascade_ctx& ctx, cudaStream_t s) {
  (void)s;
  if (ctx.blocks.size() > 1) {
    // The previous call grew the arena: fold the blocks into one so that the
    // next call of the same size needs no allocation.  Growth is rare, so a
    // device-wide wait here is acceptable.
    KS_CUDA(cudaDeviceSynchronize());
    size_t total = 0;
    for (auto& b : ctx.blocks) {
      total += b.cap;
      if (b.owned) cudaFree(b.ptr);
    }
    ctx.blocks.clear();
    char* p = nullptr;
    if (cudaMalloc(&p, total) != cudaSuccess) {
      cudaGetLastError();
      return KASCADE_ERR_OOM;
    }
    ctx.blocks.push_back({p, total, 0});
  }
  for (auto& b : ctx.blocks) b.used = 0;
  return KASCADE_OK;
}

void* arena_alloc(kascade_ctx& ctx, size_t bytes) {
  bytes = (bytes + 255) & ~size_t(255);
  if (!ctx.blocks.empty()) {
    auto& b = ctx.blocks.back();
    if (b.used + bytes <= b.cap) {
      void* p = b.ptr + b.used;
      b.used += bytes;
      return p;
    }
  }
  size_t prev = ctx.blocks.empty() ? 0 : ctx.blocks.back().cap;
  size_t cap = bytes;
  if (cap < prev) cap = prev;
  if (cap < ctx.reserve_bytes) cap = ctx.reserve_bytes;
  if (cap < (size_t(64) << 20)) cap = size_t(64) << 20;
  char* p = nullptr;
  if (cudaMalloc(&p, cap) != cudaSuccess) {
    cudaGetLastError();
    // retry with exactly what is needed
    if (cap == bytes || cudaMalloc(&p, bytes) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    cap = bytes;
  }
  ctx.blocks.push_back({p, cap, bytes, true});
  return p;
}

void arena_adopt(kascade_ctx& ctx, char* p, size_t bytes) {
  for (auto& b : ctx.blocks)
    if (b.owned) cudaFree(b.ptr);
  ctx.blocks.clear();
  ctx.blocks.push_back({p, bytes, 0, false});
  ctx.reserve_bytes = bytes;
}

cudaError_t ensure_device(int device) {
  int cur = -1;
  if (cudaGetDevice(&cur) == cudaSuccess && cur == device) return cudaSuccess;
  return cudaSetDevice(device);
}

kascade_status status_reset(kascade_ctx& ctx, cudaStream_t s) {
  KS_CUDA(cudaMemsetAsync(ctx.d_status, 0, sizeof(DevStatus), s));
  return KASCADE_OK;
}

static void collect_times(kascade_ctx& ctx) {
  for (auto& p : ctx.pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
      auto& t = ctx.times[p.name];
      t.first += ms;
      t.second += 1;
    } else {
      cudaGetLastError();
    }
    ctx.event_pool.push_back(p.a);
    ctx.event_pool.push_back(p.b);
  }
  ctx.pending.clear();
}

kascade_status status_finish(kascade_ctx& ctx, cudaStream_t s) {
  cudaError_t e = cudaMemcpyAsync(ctx.h_pinned, ctx.d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    ctx.last_status = cuda_status(e);
    return ctx.last_status;
  }
  collect_times(ctx);
  if (ctx.pending_levels) {
    const uint32_t* lv = reinterpret_cast<const uint32_t*>(ctx.h_pinned + KS_PINNED_LEVELS);
    // level 0's size: the call's n, or the device's count when only that
    // knows it (a tour sized for a bound)
    ctx.last_levels.assign(1, lv[0] ? (unsigned long long)lv[0] : ctx.pending_n);
    for (int k = 1; k <= ctx.pending_levels; ++k) ctx.last_levels.push_back(lv[k]);
    ctx.pending_levels = 0;
  }
  const DevStatus* st = reinterpret_cast<const DevStatus*>(ctx.h_pinned);
  ctx.error_info = st->info;
  ctx.last_status = (kascade_status)st->code;
  return ctx.last_status;
}

kascade_status read_u32(kascade_ctx& ctx, const uint32_t* dptr, uint32_t* out, cudaStream_t s) {
  uint32_t* hp = reinterpret_cast<uint32_t*>(ctx.h_pinned + 32);
  KS_CUDA(cudaMemcpyAsync(hp, dptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  KS_CUDA(cudaStreamSynchronize(s));
  *out = *hp;
  return KASCADE_OK;
}

static cudaEvent_t take_event(kascade_ctx& ctx) {
  if (!ctx.event_pool.empty()) {
    cudaEvent_t e = ctx.event_pool.back();
    ctx.event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return e;
}

ProfScope::ProfScope(kascade_ctx& c, const char* nm, cudaStream_t st) : ctx(c), s(st), name(nm) {
  if (!ctx.profile) return;
  b = take_event(ctx);
  if (b) cudaEventRecord(b, s);
}

ProfScope::~ProfScope() {
  if (!ctx.profile || !b) return;
  cudaEvent_t e = take_event(ctx);
  if (!e) return;
  cudaEventRecord(e, s);
  ctx.pending.push_back({name, b, e});
}

}  // namespace ks
