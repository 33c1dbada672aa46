// Shared device-side definitions of the B200 list-ranking library.
//
// Element state lives in one 16-byte record per element (`Rec`), so that the
// dependent hop of the ruler chase is a single aligned 16 B load and the
// chase's own write lands in the same 32 B sector it just read.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/kascade_b200.h"

namespace ks {

// ---------------------------------------------------------------------------
// Element record.
//   a : weight (unreached or ruler) or distance from the element's ruler
//       (reached), as 64-bit two's complement
//   b : successor index (every state keeps it)
//   c : tag -- TAG_UNREACHED, TAG_RULER | ruler id, or a ruler id (reached)
// ---------------------------------------------------------------------------
struct __align__(16) Rec {
  uint64_t a;
  uint32_t b;
  uint32_t c;
};
static_assert(sizeof(Rec) == 16, "record must be 16 bytes");

constexpr uint32_t TAG_UNREACHED = 0xFFFFFFFFu;
constexpr uint32_t TAG_RULER = 0x80000000u;
constexpr uint32_t MAX_RULERS = 0x7FFFFFFEu;  // ruler ids stay below this
constexpr uint32_t MAX_ELEMS = 0xFFFFFFFEu;   // element indices fit in 32 bits

__host__ __device__ __forceinline__ bool tag_unreached(uint32_t c) { return c == TAG_UNREACHED; }
__host__ __device__ __forceinline__ bool tag_ruler(uint32_t c) {
  return (c & TAG_RULER) != 0u && c != TAG_UNREACHED;
}
__host__ __device__ __forceinline__ uint32_t tag_id(uint32_t c) { return c & 0x7FFFFFFFu; }

// Result of a deeper level for one of its elements: rank (distance to root)
// and the root as a level-0 element index.
struct __align__(16) Out {
  uint64_t rank;
  uint32_t root;
  uint32_t pad;
};
static_assert(sizeof(Out) == 16, "Out must be 16 bytes");

// Pointer-doubling record (double-buffered jump kernel).
struct __align__(16) PdRec {
  uint64_t rank;
  uint32_t succ;
  uint32_t done;  // 1 once succ is a root
};

// ---------------------------------------------------------------------------
// Device status word: the first error wins; kernels never trap.
// ---------------------------------------------------------------------------
struct DevStatus {
  unsigned int code;
  unsigned int pad;
  unsigned long long info;
  unsigned long long counter[6];
};

__device__ __forceinline__ void set_error(DevStatus* st, unsigned int code, unsigned long long info) {
  if (atomicCAS(&st->code, 0u, code) == 0u) st->info = info;
}

// ---------------------------------------------------------------------------
// Counter hash used for ruler sampling (the "lowbias32" integer mixer,
// a public-domain construction by C. Wellons).
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

__device__ __forceinline__ bool sampled(uint32_t x, uint32_t salt, uint32_t thresh) {
  return mix32(x ^ salt) < thresh;
}

// ---------------------------------------------------------------------------
// Cache-hinted 16 B accesses.  .cg bypasses L1 (random hops never hit it and
// the chase rewrites what it reads); .cs marks streaming data evict-first.
// ---------------------------------------------------------------------------
__device__ __forceinline__ Rec ld_rec_cg(const Rec* p) {
  uint4 v = __ldcg(reinterpret_cast<const uint4*>(p));
  Rec r;
  r.a = (uint64_t)v.x | ((uint64_t)v.y << 32);
  r.b = v.z;
  r.c = v.w;
  return r;
}
__device__ __forceinline__ Rec ld_rec_cs(const Rec* p) {
  uint4 v = __ldcs(reinterpret_cast<const uint4*>(p));
  Rec r;
  r.a = (uint64_t)v.x | ((uint64_t)v.y << 32);
  r.b = v.z;
  r.c = v.w;
  return r;
}
__device__ __forceinline__ void st_rec_cg(Rec* p, Rec r) {
  uint4 v = make_uint4((uint32_t)r.a, (uint32_t)(r.a >> 32), r.b, r.c);
  __stcg(reinterpret_cast<uint4*>(p), v);
}
__device__ __forceinline__ void st_rec_cs(Rec* p, Rec r) {
  uint4 v = make_uint4((uint32_t)r.a, (uint32_t)(r.a >> 32), r.b, r.c);
  __stcs(reinterpret_cast<uint4*>(p), v);
}
__device__ __forceinline__ Out ld_out(const Out* p) {
  uint4 v = __ldcg(reinterpret_cast<const uint4*>(p));
  Out o;
  o.rank = (uint64_t)v.x | ((uint64_t)v.y << 32);
  o.root = v.z;
  o.pad = v.w;
  return o;
}
// The same load, with the line kept in L2 ahead of streaming traffic: for
// small tables read at random by every element (a level's ruler results).
__device__ __forceinline__ uint64_t l2_keep_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
// Through the read-only (L1) path with the same L2 hint: for lookups whose
// neighbours in a warp's stream tend to repeat (log entries of one chain).
__device__ __forceinline__ Out ld_out_nc_keep(const Out* p, uint64_t pol) {
  uint32_t a, b, c, d;
  asm volatile("ld.global.nc.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
               : "=r"(a), "=r"(b), "=r"(c), "=r"(d)
               : "l"(p), "l"(pol));
  Out o;
  o.rank = (uint64_t)a | ((uint64_t)b << 32);
  o.root = c;
  o.pad = d;
  return o;
}
__device__ __forceinline__ Out ld_out_keep(const Out* p, uint64_t pol) {
  uint32_t a, b, c, d;
  asm volatile("ld.global.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
               : "=r"(a), "=r"(b), "=r"(c), "=r"(d)
               : "l"(p), "l"(pol));
  Out o;
  o.rank = (uint64_t)a | ((uint64_t)b << 32);
  o.root = c;
  o.pad = d;
  return o;
}
__device__ __forceinline__ void st_out(Out* p, uint64_t rank, uint32_t root) {
  __stcg(reinterpret_cast<uint4*>(p), make_uint4((uint32_t)rank, (uint32_t)(rank >> 32), root, 0u));
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Block-wide exclusive scan of one uint32 per thread; returns the prefix and
// writes the block total to *total.  `smem` needs blockDim/32 + 1 words.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* smem, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = (lane < nwarps) ? smem[lane] : 0u;
    uint32_t t = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < nwarps) smem[lane] = t - w;
    if (lane == nwarps - 1) smem[32] = t;
  }
  __syncthreads();
  uint32_t res = smem[warp] + x - v;
  *total = smem[32];
  __syncthreads();
  return res;
}

}  // namespace ks
