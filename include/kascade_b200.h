/*
 * kascade_b200 -- list ranking and tree rooting on one NVIDIA B200 (sm_100a).
 *
 * C ABI of libkascade_b200.so.  It replaces the free functions of the
 * reference's lib/kascade (niklas-uhl/kascade) for one GPU: the MPI
 * Distribution and Communicator arguments disappear, the arrays become
 * device (or host) pointers plus a length, and errors become status codes.
 *
 * Conventions
 *  - Indices are uint64_t (reference idx_t, lib/kascade/types.hpp:8); ranks
 *    are int64_t in the reference-shaped calls (rank_t, types.hpp:9) and
 *    uint64_t in the plain calls.  A root is an element that is its own
 *    successor (lib/kascade/successor_utils.cpp:65-70).
 *  - Element counts are limited to n <= 2^32 - 2 for lists and n <= 2^31 - 1
 *    for forests (the library keeps 32-bit indices in HBM).
 *  - Device-pointer calls are ordered on `stream` (a cudaStream_t, NULL =
 *    legacy default stream).  They return once the result is complete and
 *    its status known, unless kascade_opts.async is set, in which case they
 *    return after enqueueing and kascade_ctx_sync() reports the status.
 *  - One context per host thread; contexts own all scratch memory.
 *  - No exceptions cross this boundary.
 */
#ifndef KASCADE_B200_H
#define KASCADE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define KASCADE_API
#else
#define KASCADE_API __attribute__((visibility("default")))
#endif

typedef enum kascade_status {
  KASCADE_OK = 0,
  KASCADE_ERR_INVALID_ARG = 1,  /* bad pointer / size / option                    */
  KASCADE_ERR_OUT_OF_RANGE = 2, /* a successor or parent index >= n               */
  KASCADE_ERR_CYCLE = 3,        /* a cycle without a root (a bounded loop ran out) */
  KASCADE_ERR_NOT_A_LIST = 4,   /* an element with two predecessors given to a
                                   list ranker                                   */
  KASCADE_ERR_TIMEOUT = 5,      /* a bounded device wait ran out                 */
  KASCADE_ERR_OOM = 6,          /* device or pinned allocation failed            */
  KASCADE_ERR_CUDA = 7,         /* a CUDA runtime call failed                    */
  KASCADE_ERR_TOO_LARGE = 8,    /* n beyond the supported index range            */
  KASCADE_ERR_UNSUPPORTED = 9   /* option not available in this build            */
} kascade_status;

/* Algorithms, mirroring kascade::Algorithm (lib/kascade/configuration.hpp:9-18).
 * On one GPU the message layers of the variants disappear:
 *  GATHER_CHASE, POINTER_DOUBLING, ASYNC_POINTER_DOUBLING and
 *  RMA_POINTER_DOUBLING all run the double-buffered jump kernel (they accept
 *  forests of trees as well as lists); SPARSE_RULING_SET runs the recursive
 *  ruling-set ranker (lists only). */
typedef enum kascade_algorithm {
  KASCADE_ALGO_GATHER_CHASE = 0,
  KASCADE_ALGO_POINTER_DOUBLING = 1,
  KASCADE_ALGO_ASYNC_POINTER_DOUBLING = 2,
  KASCADE_ALGO_RMA_POINTER_DOUBLING = 3,
  KASCADE_ALGO_SPARSE_RULING_SET = 4,
  KASCADE_ALGO_EULER_TOUR = 5
} kascade_algorithm;

/* Tunables.  Zero means "choose automatically" (the autotuned table).  The
 * reference's ruler-selection strategies (ruler_selection.hpp:18-79) size the
 * ruler set by the MPI rank count; on one GPU the mean ruler spacing is the
 * tunable instead (sparse_ruling_set.cpp:120-136 picks; here a counter hash
 * picks). */
typedef struct kascade_opts {
  uint32_t struct_size;       /* sizeof(kascade_opts)                               */
  uint32_t algorithm;         /* kascade_algorithm for list ranking                 */
  uint32_t ruler_spacing;     /* mean elements per ruler at level 0 (0 = auto)      */
  uint32_t ruler_spacing_deep;/* the same for recursion levels >= 1 (0 = auto)      */
  uint32_t max_levels;        /* ruling-set recursion depth before the base case
                                 (sparse_ruling_set_rounds, configuration.hpp:70)  */
  uint32_t base_case_size;    /* at most this many elements go to the one-CTA
                                 base case (0 = auto)                              */
  uint32_t chains_per_thread; /* independent chains in flight per thread (0=auto) */
  uint32_t block_size;        /* threads per CTA of the chase kernel (0 = auto)     */
  uint32_t validate;          /* 1: check is_list before a list-only algorithm      */
  uint32_t async;             /* 1: return after enqueueing; see kascade_ctx_sync   */
  uint32_t profile;           /* 1: time each kernel with CUDA events               */
  uint32_t seed;              /* ruler-sampling seed                                */
  uint32_t level0_mode;       /* first level: 0 auto (write-free from 2^25
                                 elements on, where it is faster), 1 stamping
                                 chase, 2 write-free chase (read-only chase, log,
                                 radix partition by element, dense placement);
                                 in-place calls always stamp                      */
  uint32_t max_chain;         /* hop cap of the write-free chase before it hands
                                 level 0 to the stamping chase (0 = 64 x spacing)  */
} kascade_opts;

typedef struct kascade_ctx kascade_ctx;

KASCADE_API const char* kascade_version(void);
KASCADE_API const char* kascade_status_string(kascade_status s);
KASCADE_API void kascade_opts_init(kascade_opts* opts);

/* Context: device, scratch arena (grows on demand, reused across calls),
 * status word and pinned read-back buffer. */
KASCADE_API kascade_status kascade_ctx_create(int device, kascade_ctx** out);
KASCADE_API kascade_status kascade_ctx_destroy(kascade_ctx* ctx);
/* Pre-size the scratch arena to hold `bytes` (avoids growth inside a call). */
KASCADE_API kascade_status kascade_ctx_reserve(kascade_ctx* ctx, uint64_t bytes);
/* Scratch bytes a call of that size typically needs (the arena grows beyond
 * this only for inputs made mostly of roots). */
KASCADE_API uint64_t kascade_scratch_bytes_rank_list(uint64_t n);
KASCADE_API uint64_t kascade_scratch_bytes_root_forest(uint64_t n);
/* Wait for the context's last call on `stream` and return its status. */
KASCADE_API kascade_status kascade_ctx_sync(kascade_ctx* ctx, void* stream);
/* Detail of the last device-side error (e.g. the offending index). */
KASCADE_API uint64_t kascade_ctx_error_info(kascade_ctx* ctx);
/* Kernel timings of the last profiled call(s): fills up to `cap` entries of
 * names/milliseconds/launch counts, returns the number of kernels. */
KASCADE_API int kascade_ctx_kernel_times(kascade_ctx* ctx, const char** names, double* ms,
                                         uint64_t* launches, int cap);
KASCADE_API void kascade_ctx_reset_kernel_times(kascade_ctx* ctx);
/* Per-call statistics of the last ranking (levels, rulers per level). */
KASCADE_API int kascade_ctx_last_levels(kascade_ctx* ctx, uint64_t* sizes, int cap);

/* ----------------------------------------------------------------------------
 * List ranking, plain form (device pointers).
 *   succ[i]   successor of i (succ[i] == i marks a root)
 *   weights   distance from i to succ[i] (NULL = unit); ignored at roots
 *   root_out  root of i;  rank_out: sum of weights from i to its root,
 *             excluding the root (0 at roots)
 * Replaces: set_initial_ranking_state + sparse_ruling_set / pointer_doubling
 * (lib/kascade/list_ranking.hpp:47-50, sparse_ruling_set.hpp:13-18,
 * pointer_doubling.hpp:18-23); outputs must not alias succ.
 * ------------------------------------------------------------------------- */
KASCADE_API kascade_status kascade_rank_list(kascade_ctx* ctx, const uint64_t* succ,
                                             const uint32_t* weights, uint64_t n,
                                             uint64_t* root_out, uint64_t* rank_out,
                                             const kascade_opts* opts, void* stream);

/* Host-pointer variant: copies in, ranks, copies out (pinned or pageable).
 * With kascade_opts.async set it returns once the copies and the ranking are
 * enqueued: the host buffers stay the call's (inputs unchanged, outputs
 * unread) until kascade_ctx_sync(ctx) returns.  Calls on two contexts and two
 * streams, from pinned buffers, then overlap one call's copy-out with the
 * next call's copy-in (the two PCIe directions) and its ranking. */
KASCADE_API kascade_status kascade_rank_list_host(kascade_ctx* ctx, const uint64_t* succ,
                                                  const uint32_t* weights, uint64_t n,
                                                  uint64_t* root_out, uint64_t* rank_out,
                                                  const kascade_opts* opts, void* stream);

/* ----------------------------------------------------------------------------
 * Reference-shaped in-place calls (device pointers).  succ_array holds the
 * successors on input and the roots on output; rank_array holds each
 * element's distance to its successor on input (0 at roots) and its distance
 * to the root on output.  Roots keep their input values, exactly as the
 * reference's GatherChase leaves them (local_pointer_chasing.cpp:18-59).
 * ------------------------------------------------------------------------- */
/* kascade::sparse_ruling_set (sparse_ruling_set.hpp:13-18, sparse_ruling_set.cpp:335-392) */
KASCADE_API kascade_status kascade_sparse_ruling_set(kascade_ctx* ctx, const kascade_opts* opts,
                                                     uint64_t* succ_array, int64_t* rank_array,
                                                     uint64_t n, void* stream);
/* kascade::pointer_doubling (pointer_doubling.hpp:18-23), also standing in for
 * async_pointer_doubling and rma_pointer_doubling (:29-43) */
KASCADE_API kascade_status kascade_pointer_doubling(kascade_ctx* ctx, const kascade_opts* opts,
                                                    uint64_t* succ_array, int64_t* rank_array,
                                                    uint64_t n, void* stream);
/* kascade::rank_on_root / local_pointer_chasing (list_ranking.hpp:19-28):
 * the GatherChase contract, forests of trees allowed */
KASCADE_API kascade_status kascade_rank_on_root(kascade_ctx* ctx, uint64_t* succ_array,
                                                int64_t* rank_array, uint64_t n, void* stream);
/* kascade::set_initial_ranking_state (list_ranking.hpp:47-50, list_ranking.cpp:60-80):
 * root := succ, rank := 1 (0 at roots) */
KASCADE_API kascade_status kascade_set_initial_ranking_state(kascade_ctx* ctx, const uint64_t* succ,
                                                             uint64_t* root_array,
                                                             int64_t* rank_array, uint64_t n,
                                                             void* stream);
/* kascade::is_list (successor_utils.hpp:19-24): 1 if no element has two
 * predecessors */
KASCADE_API kascade_status kascade_is_list(kascade_ctx* ctx, const uint64_t* succ, uint64_t n,
                                           int* is_list_out, void* stream);

/* ----------------------------------------------------------------------------
 * Result statistics on the device: the bench's compute_stats
 * (bench/detail/stats.hpp:9-49, bench/detail/stats.cpp:24-162) over root and
 * rank arrays (a ranking's or a rooting's output).  Level values are the
 * reference's StatsLevel.  Basic: trees = elements with root[i] == i, max and
 * mean rank.  Extensive (both levels): per tree (keyed by root) size, rank sum
 * and max rank, reduced to the counts and means below; EXTENSIVE also lists
 * the non-trivial trees (size > 1) into per_tree (device memory, up to
 * per_tree_cap entries, ordered by root; *per_tree_count = how many exist).
 * As in the reference: a tree's max_rank starts at 0 (TreeStats,
 * stats.hpp:23-27), so a tree of negative ranks reports 0; avg_rank divides
 * the rank sum taken as an unsigned 64-bit value (the std::size_t fold of
 * stats.cpp:124-137) by n.
 * ---------------------------------------------------------------------------*/
typedef enum {
  KASCADE_STATS_NONE = 1,
  KASCADE_STATS_BASIC = 2,
  KASCADE_STATS_REDUCED_EXTENSIVE = 3,
  KASCADE_STATS_EXTENSIVE = 4
} kascade_stats_level;

typedef struct kascade_stats {
  /* BasicStats */
  uint64_t num_trees;
  int64_t max_rank;
  double avg_rank;
  /* ExtensiveStats (levels 3 and 4) */
  uint64_t ext_num_trees; /* distinct roots among root[]                 */
  uint64_t num_nontrivial_trees;
  uint64_t nontrivial_size_sum;
  int64_t nontrivial_rank_sum;
  uint64_t max_size;
  double avg_size;
  double nontrivial_avg_size;
  double nontrivial_avg_rank;
} kascade_stats;

typedef struct kascade_tree_stats {
  uint64_t root;
  uint64_t size;
  int64_t max_rank;
  int64_t rank_sum;
} kascade_tree_stats;

KASCADE_API kascade_status kascade_compute_stats(kascade_ctx* ctx, const uint64_t* root, const int64_t* rank,
                                                 uint64_t n, int level, kascade_stats* out,
                                                 kascade_tree_stats* per_tree, uint64_t per_tree_cap,
                                                 uint64_t* per_tree_count, void* stream);

/* ----------------------------------------------------------------------------
 * Tree rooting (device pointers).
 *   parent[v] (parent[v] == v marks a root) -> root_out[v], depth_out[v]
 *   (edge count to the root; 0 at roots), via an Euler tour of the forest
 *   ranked by the ruling-set ranker.
 * Replaces: rank_via_euler_tour (eulertour.hpp:22-27, eulertour.cpp:337-377).
 * ------------------------------------------------------------------------- */
KASCADE_API kascade_status kascade_root_forest(kascade_ctx* ctx, const uint64_t* parent,
                                               uint64_t n, uint64_t* root_out,
                                               uint64_t* depth_out, const kascade_opts* opts,
                                               void* stream);
/* Host-pointer variant; kascade_opts.async as for kascade_rank_list_host. */
KASCADE_API kascade_status kascade_root_forest_host(kascade_ctx* ctx, const uint64_t* parent,
                                                    uint64_t n, uint64_t* root_out,
                                                    uint64_t* depth_out, const kascade_opts* opts,
                                                    void* stream);
/* In-place form of kascade::rank_via_euler_tour: succ_array holds parents on
 * input and roots on output, rank_array receives depths; roots keep their
 * input values (eulertour.cpp:249-277 writes non-roots only). */
KASCADE_API kascade_status kascade_rank_via_euler_tour(kascade_ctx* ctx, const kascade_opts* opts,
                                                       uint64_t* succ_array, int64_t* rank_array,
                                                       uint64_t n, void* stream);
/* kascade::compute_euler_tour (eulertour.hpp:32-34, eulertour.cpp:379-392) on
 * one rank: the tour's successor array in the reference's element numbering,
 * m = 2 (n - #roots) + #roots elements.  tour_succ must hold 2n entries;
 * *m_out receives m.  The high-degree proxy construction
 * (use_high_degree_handling, successor_utils.cpp:302-418) builds the same
 * tour on one rank: its proxies stand in for remote parents only. */
KASCADE_API kascade_status kascade_compute_euler_tour(kascade_ctx* ctx, const uint64_t* parent,
                                                      uint64_t n, uint64_t* tour_succ,
                                                      uint64_t* m_out, void* stream);

/* ----------------------------------------------------------------------------
 * Pack / unpack of an active sub-list (lib/kascade/pack.hpp:23-177).
 * active[] lists k element indices in increasing order; every active
 * element's successor must be active.  pack writes the sub-list in the dense
 * index space 0..k-1; unpack writes a ranked sub-list back, translating its
 * successors (roots) to original indices.
 * ------------------------------------------------------------------------- */
KASCADE_API kascade_status kascade_pack(kascade_ctx* ctx, const uint64_t* succ,
                                        const int64_t* rank, uint64_t n, const uint64_t* active,
                                        uint64_t k, uint64_t* succ_packed, int64_t* rank_packed,
                                        void* stream);
KASCADE_API kascade_status kascade_unpack(kascade_ctx* ctx, const uint64_t* succ_packed,
                                          const int64_t* rank_packed, const uint64_t* active,
                                          uint64_t k, uint64_t* succ, int64_t* rank, uint64_t n,
                                          void* stream);

/* ----------------------------------------------------------------------------
 * Seeded synthetic inputs (device pointers), the benchmark generators.
 *   layout: 0 random permutation order, 1 runs of 64 consecutive indices in
 *   random run order, 2 identity order.  kind: 0 random recursive trees in
 *   `blocks` trees, 1 caterpillars (`blocks` of them, spine length `spine`).
 * ------------------------------------------------------------------------- */
KASCADE_API kascade_status kascade_gen_list(uint64_t n, uint64_t seed, uint32_t layout,
                                            uint64_t* succ, void* stream);
KASCADE_API kascade_status kascade_gen_weights(uint64_t n, uint64_t seed, uint32_t wbits,
                                               uint32_t* weights, void* stream);
KASCADE_API kascade_status kascade_gen_forest(uint64_t n, uint64_t seed, uint32_t kind,
                                              uint64_t blocks, uint64_t spine, uint64_t* parent,
                                              void* stream);

/* ----------------------------------------------------------------------------
 * Batched ranking: many independent lists and forests in one call, ranked by
 * one shared ruler chase (one persistent launch, one device work queue).
 * Instances are concatenated in `input` (instance-local successor or parent
 * indices); segs[i] gives instance i's offset (= sum of the earlier sizes),
 * size and kind.  Outputs are written at the same positions: for lists root
 * and rank, for forests root and depth, roots relative to their instance.
 * weights (optional) apply to list instances.  Each instance's ruler spacing
 * comes from the context's size-class table unless opts->ruler_spacing is
 * set.  No counterpart in the reference (it ranks one distributed instance
 * per call).
 * ------------------------------------------------------------------------- */
#define KASCADE_SEG_LIST 0u
#define KASCADE_SEG_FOREST 1u
typedef struct kascade_segment {
  uint64_t offset;
  uint64_t size;
  uint32_t kind; /* KASCADE_SEG_LIST or KASCADE_SEG_FOREST */
  uint32_t reserved;
} kascade_segment;

KASCADE_API kascade_status kascade_rank_batch(kascade_ctx* ctx, const kascade_segment* segs,
                                              uint32_t num_segs, const uint64_t* input,
                                              const uint32_t* weights, uint64_t total_n,
                                              uint64_t* root_out, uint64_t* rank_out,
                                              const kascade_opts* opts, void* stream);

/* Size classes: an instance of at most max_size[i] elements (tour elements
 * for forests: twice the vertex count) uses mean ruler spacing spacing[i];
 * classes in increasing max_size, the last one covering everything. */
KASCADE_API kascade_status kascade_ctx_set_size_classes(kascade_ctx* ctx, const uint64_t* max_size,
                                                        const uint32_t* spacing, uint32_t count);
KASCADE_API int kascade_ctx_get_size_classes(kascade_ctx* ctx, uint64_t* max_size, uint32_t* spacing,
                                             int cap);
/* Per size class (same count and order as the size-class table): chains in
 * flight per chase thread (1, 2 or 4), chase block size (128, 256 or 512) and
 * the ruler spacing for calls that rank one instance on their own (NULL:
 * unchanged; the table's spacing applies inside batches).  A call uses the
 * class of its size; a batch the class that holds most of its elements.
 * kascade_ctx_set_size_classes resets these to 2, 256 and its own spacing. */
KASCADE_API kascade_status kascade_ctx_set_class_launch(kascade_ctx* ctx, const uint32_t* chains,
                                                        const uint32_t* block, const uint32_t* single_spacing,
                                                        uint32_t count);
KASCADE_API int kascade_ctx_get_class_launch(kascade_ctx* ctx, uint32_t* chains, uint32_t* block,
                                             uint32_t* single_spacing, int cap);
/* Size this context's grids for `sms` SMs (0 = all SMs): its persistent and
 * grid-stride kernels then hold that many SMs' worth of block slots, and
 * work on other streams (the server's latency lane) finds the rest free. */
KASCADE_API kascade_status kascade_ctx_set_sm_budget(kascade_ctx* ctx, int sms);

/* ----------------------------------------------------------------------------
 * Serving: a request loop over the batched ranker (no counterpart in the
 * reference).  Requests are admitted by HBM footprint under a budget; their
 * inputs and results stay on the device; two lanes (requests up to small_max
 * elements, and larger ones) each coalesce the admitted requests waiting when
 * they become free into one batched call, so arrivals join as memory and
 * lanes free up and both lanes' work overlaps on the device.
 * ------------------------------------------------------------------------- */
typedef struct kascade_server kascade_server;
/* Batch plans: one batch captured once as a CUDA graph (the whole
 * device-driven pipeline: record build, forest tours, every ruling-set level,
 * propagation) and replayed by one graph launch per call.  The segment table
 * and the input / weight / output pointers are fixed at creation; their
 * contents may change between launches.  Creation runs the batch once and
 * returns KASCADE_ERR_UNSUPPORTED if it needs the host-driven recursion (a
 * level outgrowing its capacity, e.g. very many roots); a launch that meets
 * that case (new contents with far more roots) returns KASCADE_ERR_TIMEOUT,
 * and kascade_rank_batch handles such a batch.  A plan owns its scratch;
 * launches of one plan are ordered on the device.  No counterpart in the
 * reference (its rounds are MPI exchanges per call). */
typedef struct kascade_batch_plan kascade_batch_plan;
KASCADE_API kascade_status kascade_batch_plan_create(int device, const kascade_segment* segs, uint32_t num_segs,
                                                     const uint64_t* input, const uint32_t* weights, uint64_t total_n,
                                                     uint64_t* root_out, uint64_t* rank_out,
                                                     const kascade_opts* opts, kascade_batch_plan** plan);
KASCADE_API kascade_status kascade_batch_plan_launch(kascade_batch_plan* plan, void* stream);
KASCADE_API kascade_status kascade_batch_plan_destroy(kascade_batch_plan* plan);

typedef struct kascade_server_config {
  uint32_t struct_size;
  int device;
  uint64_t hbm_budget_bytes;     /* admission budget (default 40 GiB)             */
  uint32_t max_batch_requests;   /* requests per batch (default 4096)             */
  uint32_t reserved;
  uint64_t max_batch_elements;   /* elements per batch, large lane (default 2^27) */
  uint64_t small_max;            /* latency lane: requests up to this many
                                    elements (default 2^20)                       */
  uint64_t small_batch_elements; /* elements per batch, latency lane (2^23)       */
  uint32_t latency_sms;          /* SMs the throughput lane leaves free while the
                                    latency lane has work (default 32): its
                                    batches then run in an SM partition (a green
                                    context) of the other SMs, rounded down to a
                                    multiple of 8; 0 = no partition             */
  uint32_t small_reserve_pct;    /* share of the budget (percent, at most 90) that
                                    only latency-lane requests may fill (default
                                    10; 0 = none): an overloaded throughput lane
                                    cannot hold back small requests' admission  */
  uint64_t result_heap_bytes;    /* device memory set aside at creation for
                                    results (default hbm_budget_bytes / 2); a
                                    batch that finds no room there allocates   */
} kascade_server_config;

typedef struct kascade_server_stats {
  uint64_t completed;
  uint64_t completed_small;
  uint64_t batches;
  uint64_t elements;
  double p50_ms, p99_ms;             /* submit-to-completion latency, all requests */
  double p50_small_ms, p99_small_ms; /* requests up to small_max elements          */
  double elements_per_s;             /* completed elements / (last completion -
                                        first submission)                         */
  double requests_per_s;
  uint64_t bytes_in_use;
  /* per lane (0 latency, 1 throughput) */
  uint64_t lane_batches[2];
  uint64_t lane_elements[2];
  double lane_busy_ms[2];      /* wall time spent running batches              */
  double lane_max_batch_ms[2]; /* longest batch                                */
  uint64_t partition_sms;      /* SMs of the throughput lane's partition (0: the
                                  driver offers none; grid budgets only)        */
  uint64_t partition_batches;  /* throughput-lane batches run in the partition  */
  uint64_t admitted_while_running;      /* requests admitted while a batch was
                                           in flight (between its start and
                                           completion)                        */
  uint64_t batches_started_overlapping; /* batches started while the other
                                           lane's batch was in flight         */
} kascade_server_stats;

KASCADE_API void kascade_server_config_init(kascade_server_config* cfg);
KASCADE_API kascade_status kascade_server_create(const kascade_server_config* cfg, kascade_server** out);
KASCADE_API kascade_status kascade_server_destroy(kascade_server* server);
/* kind: KASCADE_SEG_LIST (succ + optional weights) or KASCADE_SEG_FOREST
 * (parent array).  Host input is copied at submission; a request that does
 * not fit the budget yet waits in arrival order. */
KASCADE_API kascade_status kascade_server_submit(kascade_server* server, uint32_t kind, const uint64_t* input,
                                                 const uint32_t* weights, uint64_t n, uint64_t* request_id);
/* The same for input already in device memory: it is copied into the
 * server's batch buffer when its batch runs, so it must stay valid until the
 * request completes.  A request holds its whole footprint while it waits or
 * runs and only its result bytes (16 per element) from completion until
 * release.  Requests up to small_max elements may pass larger ones that wait
 * for memory. */
KASCADE_API kascade_status kascade_server_submit_device(kascade_server* server, uint32_t kind,
                                                        const uint64_t* input, const uint32_t* weights,
                                                        uint64_t n, uint64_t* request_id);
/* Wait for completion (timeout_s < 0: forever); returns the request status. */
KASCADE_API kascade_status kascade_server_wait(kascade_server* server, uint64_t request_id, double timeout_s);
/* Device pointers to a completed request's root and rank (or depth). */
KASCADE_API kascade_status kascade_server_result_device(kascade_server* server, uint64_t request_id,
                                                        const uint64_t** root, const uint64_t** rank);
/* Copy a completed request's results to host buffers of n entries. */
KASCADE_API kascade_status kascade_server_fetch(kascade_server* server, uint64_t request_id,
                                                uint64_t* root_out, uint64_t* rank_out);
/* Drop a completed request and its device results.  The result memory is
 * reused by later batches at once: device work that reads the pointers from
 * kascade_server_result_device must have finished before this call. */
KASCADE_API kascade_status kascade_server_release(kascade_server* server, uint64_t request_id);
KASCADE_API kascade_status kascade_server_get_stats(kascade_server* server, kascade_server_stats* out);
KASCADE_API kascade_status kascade_server_reset_stats(kascade_server* server);

/* ----------------------------------------------------------------------------
 * Sharded list ranking: one list spread over several GPUs (one process each)
 * by contiguous index ranges.  Replaces the reference's Distribution
 * (lib/kascade/distribution.hpp:16-113: shard s holds global indices
 * [offsets[s], offsets[s+1])) and its synchronous ruler chasing engine
 * (sparse_ruling_set_detail/ruler_chasing_engine.hpp:57-101: rounds of one
 * all-to-all exchange of ruler messages, local targets worked on at once).
 * These calls are one shard's device work; kascade_b200/shard.py drives the
 * rounds and exchanges over torch.distributed (NCCL over NVLink).  Protocol:
 *   1. kascade_shard_prepare: records (rec: 16 B x n_local) and rulers (roots
 *      and a counter-hash sample by global index; local ids)
 *   2. ruler_base / num_sampled from every shard's ruler count; then rounds of
 *      kascade_shard_chase (first from the shard's rulers, then from the
 *      messages received) and one all-to-all of the send buffer, until no
 *      shard sends
 *   3. kascade_shard_unreached turns unreached elements (list heads ahead of
 *      their first ruler: fixup_unreached, post_invert.hpp:195-264) into
 *      rulers; fixup_base from every shard's count; their chains are chased
 *   4. every shard gathers all chain ends and ruler elements, builds the
 *      ruler sub-list (kascade_shard_sublist) and ranks it
 *      (kascade_sparse_ruling_set, in place)
 *   5. kascade_shard_propagate writes the shard's roots (global indices) and
 *      ranks (the plain contract: 0 at roots)
 * The global list has fewer than 2^32 - 1 elements.  Messages and chain ends
 * are 16 B records; each call returns once its work and status are complete.
 * ------------------------------------------------------------------------- */
typedef struct kascade_shard_desc {
  uint64_t lo;          /* first global index of this shard                  */
  uint64_t n_local;     /* elements of this shard                            */
  uint64_t n_global;    /* elements of all shards                            */
  uint32_t num_shards;
  uint32_t self;        /* this shard's number                               */
  const uint64_t* offsets; /* device: num_shards + 1 range starts            */
  uint64_t ruler_base;  /* global id of this shard's first sampled ruler     */
  uint64_t num_sampled; /* this shard's sampled rulers (local ids below it)  */
  uint64_t fixup_base;  /* global id of this shard's first fix-up ruler      */
} kascade_shard_desc;
typedef struct kascade_shard_msg {
  uint32_t target; /* global index of the chain's next element */
  uint32_t ruler;  /* global ruler id of the chain             */
  uint64_t dist;   /* distance from the ruler to target        */
} kascade_shard_msg;
typedef struct kascade_shard_end {
  uint32_t ruler; /* global ruler id                            */
  uint32_t next;  /* the next ruler's global id (self at roots)  */
  uint64_t dist;  /* distance between them                       */
} kascade_shard_end;
KASCADE_API kascade_status kascade_shard_prepare(kascade_ctx* ctx, const kascade_shard_desc* desc,
                                                 const uint64_t* succ, const uint32_t* weights, uint64_t n_global,
                                                 uint32_t spacing, uint32_t seed, void* rec, uint32_t* ruler_elem,
                                                 uint64_t* num_rulers, void* stream);
/* Chains from start_rulers (local element indices of rulers) and from
 * incoming messages.  regions: num_shards x region_cap messages of scratch
 * (region_cap >= num_start + num_in); send receives the outgoing messages
 * grouped by destination shard, sent_counts[d] their counts; chain ends are
 * appended to ends (*num_ends in: entries so far, out: the new total). */
KASCADE_API kascade_status kascade_shard_chase(kascade_ctx* ctx, const kascade_shard_desc* desc, void* rec,
                                               const uint32_t* start_rulers, uint64_t num_start,
                                               const kascade_shard_msg* incoming, uint64_t num_in,
                                               kascade_shard_msg* regions, uint64_t region_cap,
                                               kascade_shard_msg* send, uint64_t* sent_counts,
                                               kascade_shard_end* ends, uint64_t* num_ends, uint64_t end_cap,
                                               void* stream);
/* Unreached elements become rulers with local ids first_lid.. (appended to
 * ruler_elem); *count = how many. */
KASCADE_API kascade_status kascade_shard_unreached(kascade_ctx* ctx, const kascade_shard_desc* desc, void* rec,
                                                   uint32_t* ruler_elem, uint64_t first_lid, uint64_t* count,
                                                   void* stream);
/* out[k] = lo + ruler_elem[first + k]: the global elements of local rulers. */
KASCADE_API kascade_status kascade_shard_ruler_globals(kascade_ctx* ctx, const uint32_t* ruler_elem, uint64_t lo,
                                                       uint64_t first, uint64_t count, uint64_t* out, void* stream);
/* All chain ends -> succ2[ruler] = next, w2[ruler] = distance. */
KASCADE_API kascade_status kascade_shard_sublist(kascade_ctx* ctx, const kascade_shard_end* ends, uint64_t num_ends,
                                                 uint64_t num_rulers, uint64_t* succ2, int64_t* w2, void* stream);
/* Outputs of the shard's elements from the ranked sub-list (sub_root: root
 * ruler id per ruler, sub_rank: distance to the root per ruler,
 * elem_of_ruler: global element of each ruler id). */
KASCADE_API kascade_status kascade_shard_propagate(kascade_ctx* ctx, const kascade_shard_desc* desc, const void* rec,
                                                   const uint64_t* sub_root, const int64_t* sub_rank,
                                                   const uint64_t* elem_of_ruler, uint64_t num_rulers,
                                                   uint64_t* root_out, uint64_t* rank_out, void* stream);

/* ----------------------------------------------------------------------------
 * Ranking without allocation -- no counterpart in the reference.
 * For callers that may not allocate device memory (a host framework that owns
 * all device memory through its own pool, or a latency-critical path where an
 * allocation's possible device synchronisation is not acceptable): no
 * context, no cudaMalloc/cudaFree; scratch is one fixed device array of the
 * library (2 MiB, held on every GPU that loads the library until exit).
 * Same results as kascade_rank_list (lists or forests of trees) for
 * n <= KASCADE_NOALLOC_MAX_ELEMENTS; larger n returns KASCADE_ERR_TOO_LARGE.
 * All calls share the array: calls that overlap on the GPU race, so order
 * them.  The first call on a device looks up the array's address; make it
 * before any stream capture.  Synchronises `stream` before returning.  The
 * outputs are undefined unless the status is KASCADE_OK; a CUDA error left
 * pending by earlier work returns KASCADE_ERR_CUDA and is not cleared.
 * ------------------------------------------------------------------------- */
#define KASCADE_NOALLOC_MAX_ELEMENTS 65536u
KASCADE_API kascade_status kascade_rank_list_noalloc(const uint64_t* succ, const uint32_t* weights,
                                                     uint64_t n, uint64_t* root_out,
                                                     uint64_t* rank_out, void* stream);

/* ----------------------------------------------------------------------------
 * Measurement.  Random-access calibration: G random 16 B record accesses per
 * second in an array of n_records (far larger than L2).  mode 0: independent
 * reads, 1: independent read + write back, 2: dependent chains (reads),
 * 3: dependent chains with write back; dependent chains over wider records
 * (16 B of each read): 4: 32 B records rewritten whole, 5: 64 B records
 * rewritten whole, 6: 64 B records with 16 B written back, 7: 32 B records,
 * reads only.  Diagnostic with no counterpart in the
 * reference; it measures the ceiling the ruler chase runs against.
 * ------------------------------------------------------------------------- */
KASCADE_API kascade_status kascade_calibrate_random_access(kascade_ctx* ctx, uint64_t n_records,
                                                           uint32_t mode, uint32_t blocks_per_sm,
                                                           double* gaccess_per_s);

#ifdef __cplusplus
}
#endif

#endif /* KASCADE_B200_H */
