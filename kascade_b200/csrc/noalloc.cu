// List ranking for callers that cannot allocate device memory.
//
// Some callers of this library may not call cudaMalloc or cudaFree: a host
// framework that owns every byte of device memory through its own pool and
// forbids raw allocations, or code on a latency-critical path where an
// allocation (which can synchronise the device) is not acceptable.  Every
// other entry point draws its scratch from a context's arena, which the
// context allocates on demand.  kascade_rank_list_noalloc instead keeps its
// scratch in one file-scope device array that exists as soon as the library's
// device code is loaded on a GPU, so a call allocates nothing.
//
// It is the pointer-doubling ranker (the jump rounds of the multi-block path)
// restated for that fixed scratch: at most KASCADE_NOALLOC_MAX_ELEMENTS
// elements, same results as kascade_rank_list (lists or forests of trees).
//
// Limits and rules of use:
//  - The array (2 MiB + a 256 B control block) is held by every GPU that
//    loads the library until the process exits.
//  - n above the maximum returns KASCADE_ERR_TOO_LARGE; nothing is launched.
//  - All calls share the one array and it keeps the last call's contents;
//    each call clears the control block it needs at zero.  Calls whose work
//    overlaps on the GPU (different streams, or different host threads on
//    the same device without ordering) race on the array: order them.
//  - The first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (once per device, with that device current); make
//    that first call before any stream capture.
//  - When the status is not KASCADE_OK the outputs hold partial values.  An
//    error already pending on the calling thread is reported as
//    KASCADE_ERR_CUDA and left in place.
#include <mutex>

#include "common.cuh"

#define KS_NOALLOC_MAX 65536u
static_assert(KS_NOALLOC_MAX == KASCADE_NOALLOC_MAX_ELEMENTS, "header and implementation disagree");

namespace {

constexpr unsigned kMaxRounds = 20;  // ceil(log2(65536)) + 4
constexpr size_t kBufBytes = sizeof(ks::PdRec) * KS_NOALLOC_MAX;
constexpr size_t kCtlBytes = 256;  // status code, info, per-round active counts

// [0, kBufBytes): buffer A, [kBufBytes, 2 kBufBytes): buffer B, then control
static __device__ __align__(256) unsigned char g_noalloc_scratch[2 * kBufBytes + kCtlBytes];

struct Ctl {
  unsigned int code;
  unsigned int pad;
  unsigned long long info;
  unsigned int active[kMaxRounds];
};
static_assert(sizeof(Ctl) <= kCtlBytes, "control block too small");

__device__ __forceinline__ void na_error(Ctl* ctl, unsigned int code, unsigned long long info) {
  if (atomicCAS(&ctl->code, 0u, code) == 0u) ctl->info = info;
}

__global__ void __launch_bounds__(256) k_na_init(const uint64_t* __restrict__ succ, const uint32_t* __restrict__ w,
                                                 uint32_t n, ks::PdRec* __restrict__ a, Ctl* ctl) {
  for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x) {
    uint64_t s = succ[x];
    if (s >= n) {
      na_error(ctl, KASCADE_ERR_OUT_OF_RANGE, x);
      s = x;
    }
    const bool root = (s == x);
    ks::PdRec p;
    p.rank = root ? 0ull : (w ? (uint64_t)w[x] : 1ull);
    p.succ = (uint32_t)s;
    p.done = root ? 3u : 0u;
    a[x] = p;
  }
}

__global__ void __launch_bounds__(256) k_na_round(const ks::PdRec* __restrict__ a, ks::PdRec* __restrict__ b,
                                                  uint32_t n, unsigned int* __restrict__ active) {
  unsigned int cnt = 0;
  for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x) {
    ks::PdRec e = a[x];
    if (!(e.done & 1u)) {
      const ks::PdRec t = a[e.succ];
      e.rank += t.rank;
      e.succ = t.succ;
      e.done = t.done & 1u;
      cnt += (e.done & 1u) ? 0u : 1u;
    }
    b[x] = e;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(active, cnt);
}

__global__ void __launch_bounds__(256) k_na_final(const ks::PdRec* __restrict__ a, uint32_t n,
                                                  uint64_t* __restrict__ root_out, uint64_t* __restrict__ rank_out) {
  for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x) {
    const ks::PdRec e = a[x];
    if (e.done & 2u) {
      root_out[x] = x;
      rank_out[x] = 0;
    } else {
      root_out[x] = e.succ;
      rank_out[x] = e.rank;
    }
  }
}

constexpr int kMaxDevices = 128;
std::mutex g_setup_mu;
unsigned char* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device.
kascade_status scratch_address(unsigned char** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return KASCADE_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return KASCADE_ERR_CUDA;
    }
    g_scratch_addr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_addr[dev];
  return KASCADE_OK;
}

}  // namespace

extern "C" KASCADE_API kascade_status kascade_rank_list_noalloc(const uint64_t* succ, const uint32_t* weights,
                                                                uint64_t n, uint64_t* root_out, uint64_t* rank_out,
                                                                void* stream) {
  if (n > KS_NOALLOC_MAX) return KASCADE_ERR_TOO_LARGE;
  if (n == 0) return KASCADE_OK;
  if (!succ || !root_out || !rank_out) return KASCADE_ERR_INVALID_ARG;
  // an error left pending by the caller's earlier work stays the caller's:
  // report it without clearing it, so the error checks below see only this
  // call's own
  if (cudaPeekAtLastError() != cudaSuccess) return KASCADE_ERR_CUDA;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  unsigned char* base = nullptr;
  kascade_status st = scratch_address(&base);
  if (st != KASCADE_OK) return st;
  ks::PdRec* a = reinterpret_cast<ks::PdRec*>(base);
  ks::PdRec* b = reinterpret_cast<ks::PdRec*>(base + kBufBytes);
  Ctl* ctl = reinterpret_cast<Ctl*>(base + 2 * kBufBytes);
  const uint32_t m = (uint32_t)n;
  unsigned rounds = 2;
  while ((1u << (rounds - 2)) < m) rounds++;  // ceil(log2 n) + 2 jump rounds
  if (rounds > kMaxRounds) rounds = kMaxRounds;
  const unsigned grid = (m + 255) / 256;
  if (cudaMemsetAsync(ctl, 0, sizeof(Ctl), s) != cudaSuccess) {
    cudaGetLastError();
    return KASCADE_ERR_CUDA;
  }
  k_na_init<<<grid, 256, 0, s>>>(succ, weights, m, a, ctl);
  for (unsigned r = 0; r < rounds; ++r) {
    k_na_round<<<grid, 256, 0, s>>>(a, b, m, &ctl->active[r]);
    ks::PdRec* t = a;
    a = b;
    b = t;
  }
  k_na_final<<<grid, 256, 0, s>>>(a, m, root_out, rank_out);
  if (cudaGetLastError() != cudaSuccess) return KASCADE_ERR_CUDA;
  Ctl host;  // plain host memory: the read-back allocates nothing
  if (cudaMemcpyAsync(&host, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    return KASCADE_ERR_CUDA;
  }
  if (host.code != 0) return (kascade_status)host.code;
  if (host.active[rounds - 1] != 0) return KASCADE_ERR_CYCLE;
  return KASCADE_OK;
}
