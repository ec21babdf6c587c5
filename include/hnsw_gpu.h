/*
 * hnsw_gpu.h — C ABI of the B200-native query path of the hnsw-index crate.
 *
 * Plain pointers and sizes only. Every entry point returns an hnsw_status
 * (0 = success) and never throws or aborts across the boundary; the message
 * of the last failure on the calling thread is available from
 * hnsw_last_error(). Each declaration names the reference interface it stands
 * in for (paths within the hnsw-index crate).
 *
 * Buffers: the caller owns every host buffer; they are read or written only
 * during the call. The library owns device memory per handle. Functions whose
 * name ends in _device take device pointers and a cudaStream_t passed as
 * void*, and return once the work is enqueued.
 *
 * Threading: an hnsw_gpu_index / hnsw_gpu_brute handle may be searched from
 * many host threads at once (the reference's HnswIndex is Send + Sync,
 * src/hnsw/tests.rs:82-86); each call takes its own scratch slot and stream.
 */
#ifndef HNSW_GPU_H
#define HNSW_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error kinds. Mirrors Error and FormatError (src/error.rs:9-74); the
 * values from HNSW_ERR_CUDA on are new to the device path. */
typedef enum hnsw_status {
    HNSW_OK = 0,
    HNSW_ERR_DIMENSION_MISMATCH = 1,   /* Error::DimensionMismatch */
    HNSW_ERR_INVALID_DIMENSION = 2,    /* Error::InvalidDimension */
    HNSW_ERR_NON_FINITE_VECTOR = 3,    /* Error::NonFiniteVector */
    HNSW_ERR_ZERO_VECTOR = 4,          /* Error::ZeroVector */
    HNSW_ERR_DUPLICATE_KEY = 5,        /* Error::DuplicateKey */
    HNSW_ERR_CAPACITY_EXCEEDED = 6,    /* Error::CapacityExceeded */
    HNSW_ERR_QUANTIZATION_DISABLED = 7,/* Error::QuantizationDisabled */
    HNSW_ERR_INVALID_PARAMETER = 8,    /* Error::InvalidParameter */
    HNSW_ERR_FORMAT_BAD_MAGIC = 10,    /* FormatError::BadMagic */
    HNSW_ERR_FORMAT_UNSUPPORTED_VERSION = 11, /* FormatError::UnsupportedVersion */
    HNSW_ERR_FORMAT_TRUNCATED = 12,    /* FormatError::Truncated */
    HNSW_ERR_FORMAT_CHECKSUM = 13,     /* FormatError::ChecksumMismatch */
    HNSW_ERR_FORMAT_TRAILING_BYTES = 14, /* FormatError::TrailingBytes */
    HNSW_ERR_FORMAT_INVALID = 15,      /* FormatError::Invalid(what); what = hnsw_last_error() */
    HNSW_ERR_MEMORY_LIMIT_EXCEEDED = 16, /* Error::MemoryLimitExceeded */
    HNSW_ERR_CUDA = 20,                /* a CUDA call failed */
    HNSW_ERR_OUT_OF_DEVICE_MEMORY = 21,
    HNSW_ERR_TIMEOUT = 22,             /* a bounded device wait ran out */
    HNSW_ERR_ADMISSION_REJECTED = 23,  /* no scratch slot free for a request */
    HNSW_ERR_INVALID_ARGUMENT = 24,    /* null pointer, size out of the device path's range */
    HNSW_ERR_SCRATCH_OVERFLOW = 25,    /* a query outgrew its device scratch; retried internally */
    HNSW_ERR_CANCELLED = 26            /* the request was cancelled (hnsw_gpu_cancel) */
} hnsw_status;

/* Metric tags, as in the file format (src/metric.rs:44-60). */
enum { HNSW_METRIC_L2 = 0, HNSW_METRIC_INNER_PRODUCT = 1, HNSW_METRIC_COSINE = 2 };

/* Thread-local text of the last error ("invalid field: metric", ...). */
const char* hnsw_last_error(void);

/* ------------------------------------------------------------------ */
/* HNSW index on the device                                            */
/* ------------------------------------------------------------------ */

typedef struct hnsw_gpu_index hnsw_gpu_index;

typedef struct hnsw_index_info {
    uint32_t dim, metric, m, m0, ef_construction, quantized;
    uint32_t nodes;        /* tombstones included */
    uint32_t live;         /* HnswIndex::len */
    uint32_t top_level;
    uint32_t entry;        /* entry point id, 0xFFFFFFFF if empty */
    uint64_t seed;
    double level_multiplier;
    uint64_t required_memory; /* io.rs required_memory() of the file */
    uint64_t device_bytes;    /* device memory held by the handle */
} hnsw_index_info;

/* Validates a format-v1 file with every check of HnswIndex::from_bytes /
 * from_bytes_with_limit (src/hnsw/io.rs:236-540). Host only: needs no GPU.
 * max_memory == 0 means the default limit (64 x len, at least 64 MiB,
 * io.rs:269-275). info may be NULL. */
int hnsw_validate_bytes(const uint8_t* bytes, size_t len, uint64_t max_memory, hnsw_index_info* info);

/* Loads and validates a file (as hnsw_validate_bytes), then flattens it
 * into device memory on `device`. Replaces HnswIndex::from_bytes
 * (src/hnsw/mod.rs:666-700) for the device path. `bytes` may be freed after
 * the call. */
int hnsw_gpu_index_open(const uint8_t* bytes, size_t len, uint64_t max_memory, int device,
                        hnsw_gpu_index** out);
void hnsw_gpu_index_close(hnsw_gpu_index* index);
int hnsw_gpu_index_info(const hnsw_gpu_index* index, hnsw_index_info* out);

/* Replaces the tombstone column (deleted flags per node id, 0 or 1), the
 * device-side form of HnswIndex::remove (src/hnsw/mod.rs:357-365). */
int hnsw_gpu_set_tombstones(hnsw_gpu_index* index, const uint8_t* deleted, size_t nodes);

/* Options of one search call. Mirrors SearchOptions (src/hnsw/mod.rs:56-98)
 * plus the batch arguments of search_batch (mod.rs:520-536). The reference
 * filter is a closure over keys; here it is a key bitmap: key `x` passes iff
 * x < filter_nbits and bit x is set. */
typedef struct hnsw_search_opts {
    uint32_t k;                 /* results per query (when ks == NULL) */
    uint32_t ef;                /* candidate list size (when efs == NULL); raised to k */
    const uint32_t* ks;         /* optional per-query k */
    const uint32_t* efs;        /* optional per-query ef */
    int32_t quantized;          /* SearchOptions::quantized */
    const uint64_t* filter_bits;/* optional key bitmap(s) */
    uint64_t filter_nbits;      /* bits per bitmap */
    uint64_t filter_stride;     /* words between per-query bitmaps; 0 = one shared bitmap */
    const uint8_t* filter_used; /* optional per-query flag: 0 = no filter for that query */
    uint32_t out_stride;        /* entries per query row of the outputs; 0 = max k */
    int32_t mode;               /* HNSW_MODE_* */
    const uint32_t* filter_ids; /* optional: query i uses bitmap filter_ids[i] (stride filter_stride)
                                   instead of bitmap i, so many queries can share a few filters */
    int32_t filter_by_node;     /* 0: bit = key (keys below filter_nbits); 1: bit = node id, i.e.
                                   position in the file's node order, for indexes whose keys are
                                   sparse u64 values (a closure filter evaluated once per node) */
    float exact_below;          /* selectivity planner (off at 0): a filtered query whose bitmap
                                   admits at most this fraction of the live nodes is answered by an
                                   exact scan of the admitted nodes (f32, the reference's distance
                                   order, ties by key) instead of the graph walk, as the crate's
                                   documentation advises for very selective filters
                                   (src/hnsw/mod.rs:421-425). Needs node bitmaps, or keys equal to
                                   node ids; other queries are unaffected */
    int32_t traversal;          /* HNSW_TRAVERSAL_*: how distances are computed while the graph is
                                   walked. F32 (0, default) is the reference's search, bit for bit.
                                   BF16 (1) and BF16X3 (2) compute each neighbor list's distances on
                                   the tensor cores (BF16 operands, FP32 accumulation; X3 adds the
                                   two cross terms of the hi/lo split), then re-rank the ef results
                                   with exact f32 distances, as the quantized search re-ranks its int8
                                   traversal (src/hnsw/mod.rs:494-498). Results carry exact
                                   distances; the walk may differ from the f32 one where distances
                                   nearly tie. Not combined with `quantized` */
} hnsw_search_opts;

enum {
    HNSW_TRAVERSAL_F32 = 0,
    HNSW_TRAVERSAL_BF16 = 1,
    HNSW_TRAVERSAL_BF16X3 = 2
};

enum {
    HNSW_MODE_PLAIN = 0,      /* one warp per query, one launch per call */
    HNSW_MODE_PERSISTENT = 1, /* persistent CTAs draining a device work queue */
    HNSW_MODE_AUTO = 2        /* the mode hnsw_gpu_autotune found faster for this ef (else persistent) */
};

/* Batched search: HnswIndex::search_batch / search_with / search_filtered
 * (src/hnsw/mod.rs:412-536). Host buffers. queries: nq x dim row-major.
 * Outputs: out_keys/out_dist nq x out_stride, out_count[nq] results per
 * query (sorted by distance, then key), out_status[nq] per-query status
 * (HNSW_ERR_NON_FINITE_VECTOR, HNSW_ERR_ZERO_VECTOR, ...). The return value
 * is HNSW_OK when every query succeeded, else the first failing status. */
int hnsw_gpu_search_batch(hnsw_gpu_index* index, const float* queries, size_t nq, size_t dim,
                          const hnsw_search_opts* opts, uint64_t* out_keys, float* out_dist,
                          uint32_t* out_count, int32_t* out_status);

/* Same with every pointer (queries, ks, efs, filter bits, outputs) in device
 * memory, enqueued on `stream` (a cudaStream_t; NULL = the handle's own
 * stream; cudaStreamLegacy for the legacy default stream). Returns once the
 * work is enqueued; per-query statuses are written asynchronously. opts->k
 * and opts->ef bound every per-query k and ef. Calls on one handle share one
 * scratch area and are ordered on the device in call order. */
int hnsw_gpu_search_batch_device(hnsw_gpu_index* index, const float* d_queries, size_t nq, size_t dim,
                                 const hnsw_search_opts* d_opts, uint64_t* d_keys, float* d_dist,
                                 uint32_t* d_count, int32_t* d_status, void* stream);

/* A captured launch sequence (CUDA graph) of one device-pointer search:
 * the batch shape, options and buffers are fixed at capture; the caller
 * rewrites the query buffer in place and relaunches. For small batches this
 * replaces the memset and two kernel launches with one graph launch. */
typedef struct hnsw_gpu_graph hnsw_gpu_graph;
int hnsw_gpu_graph_create(hnsw_gpu_index* index, const float* d_queries, size_t nq, size_t dim,
                          const hnsw_search_opts* d_opts, uint64_t* d_keys, float* d_dist, uint32_t* d_count,
                          int32_t* d_status, hnsw_gpu_graph** out);
int hnsw_gpu_graph_launch(hnsw_gpu_graph* graph, void* stream);
void hnsw_gpu_graph_destroy(hnsw_gpu_graph* graph);

/* Scratch geometry of the traversal kernel ("schedule"). By default the
 * library picks it per call from the batch's largest ef and the index's
 * dimension (results capacity, candidate capacity, visited-hash size, warps
 * per block chosen for the most resident warps). A fixed schedule overrides
 * that; NULL restores the automatic choice. Results do not depend on it. */
typedef struct hnsw_schedule {
    uint32_t ef_cap;          /* >= every max(ef, k) of a batch; multiple of 32, <= 1024 */
    uint32_t cand_cap;        /* candidate array entries */
    uint32_t hash_cap;        /* visited-hash entries, a multiple of 64 (at least 64) */
    uint32_t warps_per_block; /* 1..8 */
    uint32_t cold_chunks;     /* pool of the queues' cold lists, in chunks of 1024 candidates;
                                 0 = automatic (8 per node or 32 per warp). A smaller pool sends
                                 more queries to the retry and last-resort passes; results
                                 never change */
    uint32_t stage_rows;      /* 0..32: neighbor rows gathered into shared memory per round with
                                 cp.async before their distances (0 = read in place) */
    uint32_t cold;            /* 1: the fast kernel's variant that keeps candidate queues of any
                                 length (cold list), for selective filters; 0: leaner variant,
                                 overflow goes to the retry pass */
} hnsw_schedule;
int hnsw_gpu_set_schedule(hnsw_gpu_index* index, const hnsw_schedule* schedule);

/* Autotuner (no reference counterpart; the crate has no device schedule).
 * Times the search of a sample batch (host buffers, same options as
 * hnsw_gpu_search_batch) under every feasible schedule of the grid
 * mode x warps per block {1, 2, 4, 8} x visited-hash size {16, 32, 64} x
 * ef_cap (rounded up to a multiple of 64, 1024..32768 entries) x staged
 * rows, by coordinate descent from the heuristic's own choice, `reps` timed runs each after one warm-up (median,
 * CUDA events). The fastest schedule of each mode is stored in the index's
 * tuning table for the ef bucket of the sample's max(ef, k) (buckets of 32),
 * used from then on by searches in that bucket unless a fixed schedule is
 * set; HNSW_MODE_AUTO picks the faster mode. Results never depend on the
 * schedule. `entries` (optional, `cap` entries) receives every trial. */
typedef struct hnsw_tune_entry {
    hnsw_schedule schedule;
    int32_t mode;  /* HNSW_MODE_PLAIN or HNSW_MODE_PERSISTENT */
    int32_t heuristic; /* 1 for the occupancy heuristic's own choice */
    float ms;      /* median time of the sample batch */
} hnsw_tune_entry;
int hnsw_gpu_autotune(hnsw_gpu_index* index, const float* queries, size_t nq, size_t dim,
                      const hnsw_search_opts* opts, uint32_t reps, hnsw_tune_entry* entries, size_t cap,
                      size_t* written, hnsw_tune_entry* best);
/* Forgets every autotuned schedule of the index. */
int hnsw_gpu_clear_tuning(hnsw_gpu_index* index);

/* Per-query traversal counters of the last search on this thread's slot
 * (device pointer, nq x 4 u32: layer-0 distances, layer-0 expansions,
 * upper-layer distances, upper-layer list reads). Enabled by
 * hnsw_gpu_set_counters(index, 1). */
int hnsw_gpu_set_counters(hnsw_gpu_index* index, int enabled);
int hnsw_gpu_read_counters(hnsw_gpu_index* index, uint32_t* host_out, size_t nq);

/* ------------------------------------------------------------------ */
/* Request loop: continuous batching over a resident index             */
/* ------------------------------------------------------------------ */
/* No single counterpart in the reference: it serves search_with
 * (src/hnsw/mod.rs:448-455) requests that arrive one at a time. A dispatcher
 * thread batches pending requests and launches each batch on its own stream
 * as soon as one of max_inflight device scratch slots is free, so requests
 * arriving while earlier batches run join the next launch and overlap on the
 * device. Each result equals the same search run alone. */

typedef struct hnsw_gpu_server hnsw_gpu_server;

typedef struct hnsw_server_config {
    uint32_t max_batch;     /* queries per launch */
    uint32_t max_inflight;  /* launches (device scratch slots) in flight */
    uint32_t max_pending;   /* queued requests before submit is rejected */
    uint32_t max_k, max_ef; /* admission bounds (scratch sizing) */
    uint32_t linger_us;     /* how long a partial batch waits while others run */
    uint64_t filter_nbits;  /* key-bitmap width of the filter bank; 0 = no filters */
    int32_t quantized;      /* int8 traversal + exact re-rank */
    const uint64_t* filter_bank; /* host: filter_count bitmaps of ceil(filter_nbits / 64) words,
                                    copied to the device at start */
    uint32_t filter_count;
    int32_t filter_by_node; /* the bank's bitmaps are indexed by node id, not key */
    int32_t mode;           /* HNSW_MODE_* of the batches; default PERSISTENT (the device work queue
                               spreads a small batch's queries over every SM); AUTO uses the tuned mode */
} hnsw_server_config;

void hnsw_server_config_default(hnsw_server_config* cfg);
int hnsw_gpu_server_start(hnsw_gpu_index* index, const hnsw_server_config* cfg, hnsw_gpu_server** out);
/* Finishes queued and in-flight requests, then frees the server. */
void hnsw_gpu_server_stop(hnsw_gpu_server* server);
/* Non-blocking: copies the query and returns a ticket, or
 * HNSW_ERR_ADMISSION_REJECTED when the queue is full. filter_id selects a
 * bitmap of the server's filter bank (-1 = no filter). */
int hnsw_gpu_submit(hnsw_gpu_server* server, const float* query, uint32_t k, uint32_t ef, int32_t filter_id,
                    uint64_t* ticket);
int hnsw_gpu_poll(hnsw_gpu_server* server, uint64_t ticket, int* done);
/* Cancels a request. A queued request leaves the queue at once; a request
 * whose batch is already on the device runs to the end there (kernels are
 * not interrupted) and its results are discarded. Either way *cancelled = 1
 * and hnsw_gpu_wait reports HNSW_ERR_CANCELLED with no results. A request
 * that has already completed keeps its results (*cancelled = 0). The ticket
 * must still be waited for to free it. */
int hnsw_gpu_cancel(hnsw_gpu_server* server, uint64_t ticket, int* cancelled);
/* Waits up to timeout_ms; copies the results (keys/dist: k entries) and the
 * request's latency (arrival to completion, microseconds), and frees the
 * ticket. */
int hnsw_gpu_wait(hnsw_gpu_server* server, uint64_t ticket, uint32_t timeout_ms, uint64_t* keys, float* dist,
                  uint32_t* count, int32_t* status, double* latency_us);
/* Open-loop load: request i is submitted at arrival_us[i] microseconds after
 * the call starts (ascending); outputs as hnsw_gpu_wait, per request, with
 * stride max_k for keys/dist (NULL to skip). Rejected requests get status
 * HNSW_ERR_ADMISSION_REJECTED and latency -1. filter_ids (NULL = none) gives
 * each request's filter-bank entry or -1. */
int hnsw_gpu_server_replay(hnsw_gpu_server* server, const float* queries, size_t n, const double* arrival_us,
                           const uint32_t* ks, const uint32_t* efs, const int32_t* filter_ids, uint64_t* out_keys,
                           float* out_dist, uint32_t* out_count, int32_t* out_status, double* out_latency_us);
/* Launched batches and queries since start. */
int hnsw_gpu_server_stats(const hnsw_gpu_server* server, uint64_t* batches, uint64_t* queries);

/* ------------------------------------------------------------------ */
/* Exact brute-force k-NN on the device                                */
/* ------------------------------------------------------------------ */

typedef struct hnsw_gpu_brute hnsw_gpu_brute;

enum {
    HNSW_PRECISION_FP32 = 0,   /* CUDA-core FP32 in the AVX2 kernel order: bit-identical distances */
    HNSW_PRECISION_BF16 = 1,   /* tcgen05 BF16 scoring, FP32 accumulate, FP32 re-rank */
    HNSW_PRECISION_BF16X3 = 2  /* 3-term BF16 split (compensated), FP32 re-rank */
};

/* BruteForceIndex::new + insert_batch (src/brute.rs:66-115): validates and
 * prepares rows (unit length for cosine) and uploads them. keys may be NULL
 * (keys 0..n-1). */
int hnsw_gpu_brute_open(const float* vectors, const uint64_t* keys, size_t n, size_t dim, int metric,
                        int device, hnsw_gpu_brute** out);
void hnsw_gpu_brute_close(hnsw_gpu_brute* brute);

/* BruteForceIndex::search_batch (src/brute.rs:169-180): exact top-k by
 * (distance total order, key). Outputs as hnsw_gpu_search_batch with
 * out_stride = k. */
int hnsw_gpu_brute_search_batch(hnsw_gpu_brute* brute, const float* queries, size_t nq, size_t dim,
                                uint32_t k, int precision, uint64_t* out_keys, float* out_dist,
                                uint32_t* out_count, int32_t* out_status);

/* Counters of the last tensor-core search on this handle: candidates kept
 * by the scoring threshold, summed over the batch's queries. */
/* BruteForceIndex::search_filtered (src/brute.rs:131-160): the exact top-k
 * among the rows a filter admits, computed in FP32 in the reference kernel
 * order (bit-identical to the reference). A row is admitted when its bit is
 * set: bit = key (keys below nbits), or the row's index in insertion order
 * with by_row (any u64 key set). One shared bitmap (stride 0), one per query
 * (stride words apart), or a bank selected per query by ids; used[q] == 0
 * turns the filter off for query q. k is capped at the index size, as in the
 * reference, and a query returns fewer results when fewer rows pass. */
typedef struct hnsw_brute_filter {
    const uint64_t* bits;
    uint64_t nbits;
    uint64_t stride;
    const uint8_t* used;
    const uint32_t* ids;
    int32_t by_row;
} hnsw_brute_filter;
int hnsw_gpu_brute_search_filtered(hnsw_gpu_brute* brute, const float* queries, size_t nq, size_t dim, uint32_t k,
                                   const hnsw_brute_filter* filter, uint64_t* out_keys, float* out_dist,
                                   uint32_t* out_count, int32_t* out_status);

typedef struct hnsw_brute_stats {
    uint64_t candidates;
    uint64_t queries;
    float prep_ms;      /* query validation, norms, BF16 split */
    float sample_ms;    /* dense scoring of the threshold sample + its select */
    float score_ms;     /* candidate scoring over all rows (the GEMM) */
    float rerank_ms;    /* candidate threshold + exact FP32 re-rank */
} hnsw_brute_stats;
int hnsw_gpu_brute_stats(const hnsw_gpu_brute* brute, hnsw_brute_stats* out);

/* Limits of the tensor-core pipeline's waits (BF16 / BF16x3 searches). Every
 * wait of the scoring kernel on its shared-memory barriers gives up after
 * `budget_cycles` SM clock cycles (0 restores the default, about 2 s): the
 * kernel then records the failure, lets its copies and MMAs finish, frees its
 * tensor memory and returns, and the search returns HNSW_ERR_TIMEOUT with the
 * handle still usable. `inject_stall` != 0 makes the MMA issuer first wait on
 * a barrier that nothing arrives at, so that wait runs out: a switch for
 * testing the timeout path without faulting the GPU (0 in normal use). No
 * counterpart in the reference (CPU-only; its errors are src/error.rs). */
int hnsw_gpu_brute_set_wait_limits(hnsw_gpu_brute* brute, uint64_t budget_cycles, int inject_stall);

/* Tensor-core kernel shape for BF16 / BF16x3 searches: 0 = one CTA per
 * 128 x 256 output tile; 1 = the two CTAs of a cluster share a 256 x 256
 * tile (tcgen05.mma with cta_group::2: each CTA loads its 128 queries and
 * half of the 256 base rows, so a K step moves a third fewer bytes per
 * product and the ring holds more of them). Results are the same either
 * way. No counterpart in the reference. */
int hnsw_gpu_brute_set_pairs(hnsw_gpu_brute* brute, int enabled);

/* Test hook: the next `count` device allocations the library attempts fail
 * as cudaErrorMemoryAllocation would, so callers can exercise the
 * HNSW_ERR_OUT_OF_DEVICE_MEMORY paths (0 clears it). The failing call leaves
 * its handle as it was; later calls allocate normally. Process-wide. No
 * counterpart in the reference. */
void hnsw_gpu_debug_fail_allocations(int count);

/* Tuning and test hook for the visited hash of the traversal kernels. By
 * default (mode 0) a power-of-two hash over an index whose node ids need at
 * most 10 bits more than the hash's log2 stores 16-bit tags (a slot holds
 * the id's low bits beside its probe distance; half the shared memory of
 * 32-bit ids, so more warps fit on an SM). mode -1 stores 32-bit ids
 * always; mode k > 0 treats ids as k bits wide at least, which leaves fewer
 * bits for probe distances, so tests can reach the path where a probe is
 * longer than a tag records (the set then moves to the warp's spill bitmap,
 * or the query to the retry pass). Results are identical in every mode.
 * Process-wide; applies to searches enqueued after the call. No counterpart
 * in the reference. */
void hnsw_gpu_debug_visit_tags(int mode);

/* Bounds checks of the checked build (libhnsw_gpu_checked.so, compiled with
 * HNSW_DEVICE_CHECKS): the traversal kernels check node ids, array
 * capacities, cold-list chunks and output rows before each use; the first
 * violation writes its site (nonzero) and the offending value into the
 * index's check word, and the access is skipped instead of faulting.
 * hnsw_gpu_check_word copies that word (site, value) and clears it when
 * `clear` is set; the normal build returns zeros. hnsw_gpu_checked_build
 * returns 1 in the checked build, else 0. No counterpart in the reference. */
int hnsw_gpu_check_word(hnsw_gpu_index* index, uint32_t out[2], int clear);
int hnsw_gpu_checked_build(void);

/* Allocation-free variant of hnsw_gpu_brute_search_batch, FP32 precision,
 * for callers that cannot allocate device memory while they run: code on a
 * latency-critical path, in a process whose memory policy forbids cudaMalloc
 * after start-up, or any caller that must not synchronise the device, which
 * cudaMalloc and cudaFree may do. It has no counterpart in the reference.
 * Inputs and outputs are device pointers the caller owns (queries nq x dim;
 * keys/dist nq x k; count and status nq). Scratch comes from one fixed
 * 8 MiB array in the library's device memory, held by every GPU that loads
 * the library until the process exits; a batch must satisfy
 *   round_up(nq * 4 * round_up(dim, 32), 256) + nq * 8 * max(1, min(k, n))
 *     <= 8 MiB (8388608 bytes),
 * otherwise the call returns HNSW_ERR_INVALID_ARGUMENT without launching
 * (n = rows in the index; the first term holds the prepared queries, the
 * second one top-k list per query and row slice, at least one slice). The
 * first call on a device looks up the array's device address (once per
 * device, with that device current); make that first call before any stream
 * capture. All calls share the one array, so calls whose work overlaps on
 * the GPU (different streams, no ordering between them) race and corrupt
 * each other's results; order them on one stream. Enqueued on `stream`;
 * NULL means the handle's own stream, which is NOT ordered with the caller's
 * streams (the legacy default stream included): a caller passing NULL must
 * finish writing d_queries first (e.g. synchronise its stream) and must
 * synchronise the device before reading the outputs. Pass cudaStreamLegacy
 * ((void*)1) to order the call with the legacy default stream. Returns once
 * enqueued. */
int hnsw_gpu_brute_search_batch_noalloc(hnsw_gpu_brute* brute, const float* d_queries, size_t nq, size_t dim,
                                        uint32_t k, uint64_t* d_keys, float* d_dist, uint32_t* d_count,
                                        int32_t* d_status, void* stream);

/* ------------------------------------------------------------------ */
/* Host-side index construction (produces format-v1 files)             */
/* ------------------------------------------------------------------ */

typedef struct hnsw_builder hnsw_builder;

typedef struct hnsw_params {
    uint32_t m, m0, ef_construction;
    double level_multiplier;
    uint32_t selection;          /* 0 = simple, 1 = heuristic */
    uint32_t extend_candidates;  /* heuristic flags */
    uint32_t keep_pruned;
    uint64_t seed;
} hnsw_params;

/* HnswParams::new(m) defaults (src/params.rs:78-87). */
void hnsw_params_default(uint32_t m, hnsw_params* out);

/* HnswIndex::new (src/hnsw/mod.rs:181-187). */
int hnsw_builder_new(size_t dim, int metric, const hnsw_params* params, hnsw_builder** out);
void hnsw_builder_free(hnsw_builder* b);
/* HnswIndex::insert (mod.rs:290-302): sequential, deterministic. */
int hnsw_builder_insert(hnsw_builder* b, uint64_t key, const float* vector, size_t dim);
/* HnswIndex::insert_batch (mod.rs:318-349): parallel link on `threads`
 * host threads (0 = all cores). */
int hnsw_builder_insert_batch(hnsw_builder* b, const uint64_t* keys, const float* vectors, size_t n,
                              size_t dim, int threads);
/* HnswIndex::remove (mod.rs:357-365). *removed = 1 if the key was live. */
int hnsw_builder_remove(hnsw_builder* b, uint64_t key, int* removed);
/* HnswIndex::compact (mod.rs:381-400): rebuilds from the live nodes with
 * link_parallel on `threads` host threads (0 = all cores). No-op without
 * tombstones. */
int hnsw_builder_compact(hnsw_builder* b, int threads);

/* Device construction. The batch is validated and appended exactly as by
 * hnsw_builder_insert_batch (same errors, index unchanged on error); the
 * new nodes are then linked on `device` in waves: every node of a wave
 * searches the graph as it stood before the wave, and its reverse edges are
 * applied list by list in ascending node id with connect's push-or-shrink
 * rule. Node levels and the wave plan depend only on the inputs, so the
 * graph is deterministic; with max_wave = 1 every wave is one node and the
 * graph equals the sequential insert() sequence bit for bit. */
typedef struct hnsw_gpu_build_opts {
    double wave_fraction; /* nodes per wave = max(1, floor(linked * fraction)); (0, 1] */
    uint32_t max_wave;    /* at most this many nodes per wave (>= 1) */
    uint32_t hash_cap;    /* visited-hash entries per warp; 0 = 16 per unit of ef */
    uint32_t timing;      /* 1 = record per-phase device times in the stats */
} hnsw_gpu_build_opts;
typedef struct hnsw_gpu_build_stats {
    uint32_t waves, nodes;
    uint64_t spills;   /* layer searches whose visited set moved to HBM */
    uint64_t inexact;  /* candidate queues that dropped a live entry (0 in practice) */
    uint64_t shrinks;  /* full lists re-selected by a reverse edge */
    uint64_t records;  /* reverse edges */
    double device_ms;  /* device time of the waves (CUDA events) */
    double search_ms, connect_ms; /* per phase, when opts.timing */
    uint64_t dist_search;  /* distances of the layer searches */
    uint64_t dist_select;  /* row pairs compared by the neighbor selections */
    uint64_t dist_connect; /* distances of the connect step (owner-member and pairs) */
    uint64_t lists0, listsU; /* neighbor lists read on layer 0 / above */
    uint32_t search_warps_per_block, search_blocks_per_sm;
    uint32_t connect_warps_per_block, connect_blocks_per_sm;
    uint32_t hash_cap;
} hnsw_gpu_build_stats;
/* Defaults: wave_fraction 0.05, max_wave 65536, hash_cap 0, timing 0. */
void hnsw_gpu_build_opts_default(hnsw_gpu_build_opts* out);
/* HnswIndex::insert_batch (mod.rs:318-338) with the link step on a GPU.
 * opts may be NULL (defaults). */
int hnsw_builder_insert_batch_gpu(hnsw_builder* b, const uint64_t* keys, const float* vectors, size_t n,
                                  size_t dim, int device, const hnsw_gpu_build_opts* opts);
/* HnswIndex::compact with the link step on a GPU. */
int hnsw_builder_compact_gpu(hnsw_builder* b, int device, const hnsw_gpu_build_opts* opts);
/* Figures of the builder's last device link (zeros before the first). */
int hnsw_builder_gpu_stats(const hnsw_builder* b, hnsw_gpu_build_stats* out);
/* HnswIndex::enable_quantization (mod.rs:544-547). */
int hnsw_builder_enable_quantization(hnsw_builder* b);
/* HnswIndex::to_bytes (mod.rs:639-643). Free the buffer with hnsw_bytes_free. */
int hnsw_builder_to_bytes(const hnsw_builder* b, uint8_t** out, size_t* len);
void hnsw_bytes_free(uint8_t* p);

/* ------------------------------------------------------------------ */
/* Synthetic data (src/synthetic.rs:81-124)                            */
/* ------------------------------------------------------------------ */

/* Dataset::gaussian: base then queries from one SplitMix64 stream. */
void hnsw_synthetic_gaussian(size_t n_base, size_t n_query, size_t dim, uint64_t seed, float* base,
                             float* queries);
/* Dataset::clustered with the spread (sigma) as a parameter: centers first,
 * then per point next_below(clusters) and dim Gaussians. */
void hnsw_synthetic_mixture(size_t n_base, size_t n_query, size_t dim, size_t clusters, double sigma,
                            uint64_t seed, float* base, float* queries);
/* The same mixture with the queries drawn from their own stream: centers
 * and base points from SplitMix64(base_seed) as hnsw_synthetic_mixture,
 * then queries (next_below(clusters) and dim Gaussians each) from
 * SplitMix64(query_seed) around the same centers. */
void hnsw_synthetic_mixture_split(size_t n_base, size_t n_query, size_t dim, size_t clusters, double sigma,
                                  uint64_t base_seed, uint64_t query_seed, float* base, float* queries);
/* CRC-32 (IEEE) of a buffer (src/crc32.rs). */
uint32_t hnsw_crc32(const uint8_t* bytes, size_t len);

#ifdef __cplusplus
}
#endif
#endif /* HNSW_GPU_H */
