// Library context: device properties, a growable scratch arena, the device
// status word, a pinned read-back buffer and optional per-kernel timing.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <map>
#include <string>
#include <vector>

#include "common.cuh"
#include "tuned_classes.h"

struct kascade_ctx {
  int device = 0;
  int sm_count = 148;
  size_t l2_bytes = 0;
  size_t smem_optin = 0;
  ks::DevStatus* d_status = nullptr;
  unsigned long long* h_pinned = nullptr;  // KS_PINNED_WORDS words
  // scratch arena: blocks are never freed inside a call, so pointers handed
  // out by alloc() stay valid until the next begin_call()
  struct Block {
    char* ptr;
    size_t cap;
    size_t used;
    bool owned = true;  // false: memory lent by the caller (arena_adopt)
  };
  std::vector<Block> blocks;
  size_t reserve_bytes = 0;
  // profiling
  bool profile = false;
  struct Pending {
    const char* name;
    cudaEvent_t a, b;
  };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> event_pool;
  std::map<std::string, std::pair<double, unsigned long long>> times;
  std::vector<std::string> time_names;  // stable storage for returned names
  std::vector<unsigned long long> last_levels;
  // level sizes of a device-driven recursion, copied to the pinned buffer by
  // the call and read into last_levels when its status is read
  int pending_levels = 0;
  unsigned long long pending_n = 0;
  unsigned long long error_info = 0;
  kascade_status last_status = KASCADE_OK;
  // ordering between calls issued on different streams: the next call's
  // stream waits for the previous call's completion event before it reuses
  // the arena
  cudaEvent_t done_event = nullptr;
  cudaStream_t last_stream = nullptr;
  bool async_pending = false;
  // an async host-buffer call ranked by the device-driven recursion: what
  // kascade_ctx_sync needs to rank it again on the host-driven path when a
  // level outgrew that recursion (the host buffers are the call's until then)
  struct HostRerun {
    bool set = false;
    int kind = 0;                     // 0: kascade_rank_list_host, 1: kascade_root_forest_host
    const uint64_t* succ = nullptr;  // successors, or parents
    const uint32_t* weights = nullptr;
    unsigned long long n = 0;
    uint64_t* root_out = nullptr;
    uint64_t* rank_out = nullptr;  // ranks, or depths
    kascade_opts opts{};
    cudaStream_t stream = nullptr;
  } host_rerun;
  // size classes: instances of at most class_max[i] elements use a mean ruler
  // spacing of class_spacing[i] inside a batch; a call (or a batch, by the class holding
  // most of its elements) chases with class_chains[i] chains per thread in
  // blocks of class_block[i] threads.  Defaults: the autotuner's table.
  std::vector<unsigned long long> class_max = KS_TUNED_MAX;
  std::vector<uint32_t> class_spacing = KS_TUNED_SPACING;
  std::vector<uint32_t> class_chains = KS_TUNED_CHAINS;
  std::vector<uint32_t> class_block = KS_TUNED_BLOCK;
  // spacing for a call that ranks one instance on its own: fewer, larger
  // levels pay off there, since each level costs launches and a host wait
  std::vector<uint32_t> class_spacing_single = KS_TUNED_SPACING_SINGLE;
  int class_of(unsigned long long n) const {
    for (size_t i = 0; i < class_max.size(); ++i)
      if (n <= class_max[i]) return (int)i;
    return (int)class_max.size() - 1;
  }
  // SMs' worth of block slots this context's kernels may occupy (0 = all):
  // grids are sized for this many SMs, so that work on other streams (a
  // server's latency lane) always finds free slots.  Read at every launch;
  // another thread may change it between launches.
  std::atomic<int> sm_budget{0};
  int usable_sms() const {
    const int b = sm_budget.load(std::memory_order_relaxed);
    return (b > 0 && b < sm_count) ? b : sm_count;
  }
};

namespace ks {

constexpr int KS_PINNED_WORDS = 64;
constexpr int KS_PINNED_LEVELS = 40;  // first word of the device-driven level sizes

// Arena -------------------------------------------------------------------
kascade_status arena_begin_call(kascade_ctx& ctx, cudaStream_t s);
// Use `bytes` of caller-owned device memory as the arena (the caller frees
// it after the context); contexts that never run concurrently may share one.
void arena_adopt(kascade_ctx& ctx, char* p, size_t bytes);
// Make `device` current unless the current context already belongs to it
// (which keeps a context the caller made current, e.g. an SM partition).
cudaError_t ensure_device(int device);
void* arena_alloc(kascade_ctx& ctx, size_t bytes);  // nullptr on OOM
template <class T>
T* alloc(kascade_ctx& ctx, size_t count) {
  return reinterpret_cast<T*>(arena_alloc(ctx, count * sizeof(T) + 16));
}

// Status --------------------------------------------------------------------
kascade_status cuda_status(cudaError_t e);
// Clear the device status word (stream-ordered).
kascade_status status_reset(kascade_ctx& ctx, cudaStream_t s);
// Synchronise `s`, read the device status word, collect kernel timings.
kascade_status status_finish(kascade_ctx& ctx, cudaStream_t s);
// Read one device word into the pinned buffer and wait for it.
kascade_status read_u32(kascade_ctx& ctx, const uint32_t* dptr, uint32_t* out, cudaStream_t s);

// Profiling ----------------------------------------------------------------
struct ProfScope {
  kascade_ctx& ctx;
  cudaStream_t s;
  const char* name;
  cudaEvent_t b = nullptr;
  ProfScope(kascade_ctx& c, const char* nm, cudaStream_t st);
  ~ProfScope();
};

inline unsigned grid_for(const kascade_ctx& ctx, uint64_t work, unsigned block, unsigned per_sm_cap) {
  uint64_t g = (work + block - 1) / block;
  uint64_t cap = (uint64_t)ctx.usable_sms() * per_sm_cap;
  if (g > cap) g = cap;
  if (g == 0) g = 1;
  return (unsigned)g;
}

}  // namespace ks

#define KS_CHECK_LAUNCH()                                   \
  do {                                                      \
    cudaError_t _e = cudaGetLastError();                    \
    if (_e != cudaSuccess) return ks::cuda_status(_e);      \
  } while (0)

#define KS_TRY(expr)                                        \
  do {                                                      \
    kascade_status _s = (expr);                             \
    if (_s != KASCADE_OK) return _s;                        \
  } while (0)

#define KS_CUDA(expr)                                       \
  do {                                                      \
    cudaError_t _e = (expr);                                \
    if (_e != cudaSuccess) return ks::cuda_status(_e);      \
  } while (0)
