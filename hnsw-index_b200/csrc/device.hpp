// Device-resident index and the launch interface of the search kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace hnswgpu {

constexpr uint32_t kSentinel = 0xFFFFFFFFu;

// Flattened HNSW index in HBM. Rows of vectors are padded to a multiple of 32
// floats (128 B), int8 code rows to a multiple of 16 bytes (zero fill, so
// integer dot products and norms are unchanged), neighbor rows to a multiple
// of 32 ids with kSentinel after the live prefix.
struct DeviceIndexView {
    uint32_t n = 0, dim = 0, dp = 0, dc = 0;
    uint32_t m = 0, m0 = 0, mp = 0, m0p = 0;
    uint32_t top = 0, entry = kSentinel, live = 0;
    int metric = 0;
    int quantized = 0;
    int keys_are_ids = 0;
    int has_dead = 0;  // any tombstone set
    float scale = 1.0f;
    const float* vec = nullptr;        // n * dp
    const int8_t* codes = nullptr;     // n * dc
    const int32_t* code_norm = nullptr;// n  (sum of squared codes)
    const float* q_offset = nullptr;   // dp (quantizer offsets)
    const uint32_t* adj0 = nullptr;    // n * m0p
    const uint32_t* up_off = nullptr;  // n: block index of the node's layer-1 list
    const uint32_t* adjU = nullptr;    // blocks * mp
    const uint64_t* keys = nullptr;    // n
    const uint32_t* dead = nullptr;    // ceil(n/32) tombstone bitmap
    // Tensor-core traversal: BF16 copies of the rows, dt (dim rounded up to
    // 32) values per node, permuted within each 32-value block so that lane
    // t of an mma quad finds its operand words in one 16-byte load
    // (tc_row_pos); the low parts of the hi/lo split; the f32 squared norms.
    const uint4* tc_hi = nullptr;      // n * dt / 8
    const uint4* tc_lo = nullptr;      // n * dt / 8 (BF16X3 only)
    const float* xnorm = nullptr;      // n
    uint32_t dt = 0;
};

// Per-launch scratch geometry (picked by the launcher per call).
struct SearchGeometry {
    uint32_t ef_cap = 64;     // results capacity (>= every ef of the batch)
    uint32_t cand_cap = 160;  // candidate queue capacity
    uint32_t hash_cap = 4096; // visited hash entries (multiple of 64)
    uint32_t warps_per_block = 4;
    uint32_t bytes_per_warp = 0;
    uint32_t cold_chunks = 0;  // cold-list pool size in chunks; 0 = automatic
    // Staged gathers: up to stage_rows fresh neighbor rows per round are
    // copied into shared memory with cp.async before their distances are
    // computed (0 = rows are read from global memory group by group).
    uint32_t stage_rows = 0;
    uint32_t stage_row_bytes = 0;  // set per launch: dc (int8 traversal) or dp * 4
    uint32_t tc_bytes = 0;         // set per launch: the query's BF16 operands (tensor-core traversal)
    // Fast-kernel variant with the cold candidate list (persistent warps
    // move queue overflow there directly instead of to a global array).
    uint32_t cold = 0;
    // Visited hash of 16-bit tags instead of 32-bit ids (set per launch by
    // set_hash_tags from the node count): half the shared memory, so more
    // warps fit on an SM. tag_sh = id bits kept in a tag, tag_mask = the id
    // space 2^B - 1.
    uint32_t tag16 = 0, tag_sh = 0, tag_mask = 0;
};

// 16-bit visited tags apply when the hash has 2^b entries (b >= 6) and node
// ids below n need B = max(b, ceil(log2 n)) bits with B - b <= 10: the id is
// mapped by a bijection of [0, 2^B), its home slot is the top b bits, and a
// tag holds the low B - b bits beside the probe distance from home (at least
// 6 bits, so probes up to 62 long). Otherwise the hash stores 32-bit ids.
// `min_bits` > 0 widens the id space (any B >= the ids' bits is exact; a
// wider one leaves fewer distance bits, down to 1, i.e. probes of length 1:
// a test setting), negative turns the tags off.
inline void set_hash_tags(SearchGeometry& g, uint32_t n, int min_bits = 0) {
    g.tag16 = g.tag_sh = g.tag_mask = 0;
    const uint32_t cap = g.hash_cap;
    if (min_bits < 0 || cap < 64 || (cap & (cap - 1)) != 0) return;
    const uint32_t b = 31u - uint32_t(__builtin_clz(cap));
    uint32_t B = n > 1 ? 32u - uint32_t(__builtin_clz(n - 1)) : 1u;
    if (B < uint32_t(min_bits)) B = uint32_t(min_bits > 32 ? 32 : min_bits);
    if (B < b) B = b;
    if (B - b > (min_bits > 0 ? 15u : 10u)) return;
    g.tag16 = 1;
    g.tag_sh = B - b;
    g.tag_mask = B >= 32 ? 0xFFFFFFFFu : (1u << B) - 1u;
}

struct SearchArgs {
    DeviceIndexView ix;
    const float* queries = nullptr;  // nq * dim
    uint32_t nq = 0;
    uint32_t k = 10, ef = 64;
    const uint32_t* ks = nullptr;
    const uint32_t* efs = nullptr;
    int quantized = 0;
    const uint64_t* filter_bits = nullptr;
    uint64_t filter_nbits = 0;
    uint64_t filter_stride = 0;
    const uint8_t* filter_used = nullptr;
    const uint32_t* filter_ids = nullptr;  // optional bitmap index per query
    int filter_by_node = 0;                // bitmaps indexed by node id instead of key
    uint64_t* out_keys = nullptr;
    float* out_dist = nullptr;
    uint32_t* out_count = nullptr;
    int32_t* out_status = nullptr;
    uint32_t out_stride = 10;
    uint32_t* counters = nullptr;  // optional nq * 4
    // Work distribution: persistent mode drains work_next; the overflow
    // list collects queries that outgrew the fast scratch.
    uint32_t* work_next = nullptr;
    uint32_t* overflow_list = nullptr;
    uint32_t* overflow_count = nullptr;
    int persistent = 0;
    // Fallback workspaces in global memory (retry kernel only).
    uint64_t* g_results = nullptr;
    uint64_t* g_cands = nullptr;
    uint32_t* g_visited = nullptr;  // bitmap, ceil(n/32) words per warp
    uint32_t g_ef_cap = 0, g_cand_cap = 0;
    uint64_t g_visited_words = 0;
    // Per-warp spill areas of the persistent kernel (slot = global warp index).
    uint32_t* spill_bits = nullptr;   // spill_slots * spill_words (multiple of 4 words)
    uint32_t spill_words = 0;
    uint64_t* spill_cands = nullptr;  // spill_slots * (spill_cand_cap + 1)
    uint32_t spill_cand_cap = 0;
    uint32_t spill_slots = 0;
    // Cold candidate lists: chunks of kColdChunk entries drawn from a pool by
    // the persistent warps of the cold variant (slot < cold_slots) and by the
    // retry warps. Each warp records the chunks it owns in its row of
    // `cold_tab` (cold_tab_cap ids). cold_next[0] counts the chunks handed
    // out by the fast kernel, cold_next[1] those of the retry kernel (which
    // reuses the whole pool).
    uint64_t* cold_pool = nullptr;
    uint32_t cold_chunks = 0;
    uint32_t* cold_next = nullptr;
    uint32_t* cold_tab = nullptr;
    uint32_t cold_tab_cap = 0;
    uint32_t cold_slots = 0;
    // Last-resort pass: the retry kernel lists the queries that still did not
    // fit (pool exhausted) here; a final launch of a few warps, each owning a
    // private region of every chunk a list can need (cold_private: the chunk
    // table rows are preassigned), runs them.
    uint32_t* overflow_list2 = nullptr;
    uint32_t* overflow_count2 = nullptr;
    int cold_private = 0;
    // Selectivity planner: planned[q] != 0 sends query q to the exact scan
    // of its admitted nodes; plan_max is the admitted-count bound.
    const uint8_t* planned = nullptr;
    uint32_t plan_max = 0;
    // Distances while walking the graph: 0 f32 (the reference's), 1 BF16
    // and 2 BF16x3 on the tensor cores with an exact f32 re-rank.
    int traversal = 0;
    // Outputs live in mapped host memory and each query's status is its
    // completion flag: the status is written last, after a system-scope
    // fence, so a host thread that sees it can read the query's results.
    int publish = 0;
    // Checked builds (HNSW_DEVICE_CHECKS): the first violated bounds check
    // writes its site into chk[0] and the offending value into chk[1], and
    // the access is skipped; unused otherwise.
    uint32_t* chk = nullptr;
};

// Kernels of the tensor-core traversal (search_tc.cu): variant v (0 lean,
// 1 cold list, 2 single array) and the retry pass, for traversal 1 (BF16)
// or 2 (BF16x3); and the builder of the BF16 rows and f32 squared norms.
using SearchKernel = void (*)(SearchArgs, SearchGeometry);
using RetryKernel = void (*)(SearchArgs);
SearchKernel tc_search_kernel(int v, int traversal, bool persistent);
RetryKernel tc_retry_kernel(int traversal);
cudaError_t launch_tc_rows(const float* vec, uint32_t n, uint32_t dim, uint32_t dp, uint32_t dt, uint4* hi, uint4* lo,
                           float* xnorm, cudaStream_t stream);

// Bytes of a warp's BF16 query operands for the tensor-core traversal.
__host__ __device__ inline uint32_t tc_query_bytes(const SearchArgs& a) {
    return a.traversal ? a.ix.dt * 2u * (a.traversal == 2 ? 2u : 1u) : 0u;
}

constexpr uint32_t kLastResortWarps = 4;

constexpr uint32_t kColdChunkShift = 10;
constexpr uint32_t kColdChunk = 1u << kColdChunkShift;  // entries per cold chunk (8 KB)

// Launches the fast search (plain or persistent) followed by the retry pass
// for queries that overflowed. All on `stream`.
cudaError_t launch_search(const SearchArgs& args, const SearchGeometry& geo, int num_sms, cudaStream_t stream);
// Selectivity planner: sets planned[q] when query q's filter admits at most
// args.plan_max nodes (counting stops early past the bound).
cudaError_t launch_plan(const SearchArgs& args, uint8_t* planned, cudaStream_t stream);
// Retry pass only (global-memory scratch); `warps` warps.
cudaError_t launch_search_retry(const SearchArgs& args, uint32_t warps, cudaStream_t stream);
// Scratch bytes per warp of a geometry for dimension dp (floats) / dc (bytes).
uint32_t geometry_bytes_per_warp(const SearchGeometry& g, uint32_t dp, uint32_t dc);
// Resident warps of the persistent kernel for a geometry (spill slots needed).
cudaError_t persistent_warps(const SearchGeometry& g, uint32_t dp, uint32_t dc, int num_sms, uint32_t* warps);

// Device ingest of a format-v1 file (ingest.cu).
constexpr size_t kIngestCrcChunk = 4096;  // bytes per CRC chunk (multiple of 16)
// CRC-32 of data[0, len) (the file buffer, 256-byte aligned) into *crc
// (host), synchronising the stream. Device scratch: part holds one word per
// chunk, pow8 64 words, out one word.
cudaError_t ingest_crc(const uint8_t* data, size_t len, uint32_t* part, uint32_t* pow8, uint32_t* out,
                       uint32_t* crc, cudaStream_t stream);
// Vector checks over the padded rows; *first = min(node * 2 + kind).
cudaError_t ingest_check_vectors(const float* vec, uint32_t n, uint32_t dim, uint32_t dp, bool cosine,
                                 unsigned long long* first, cudaStream_t stream);
// List checks and CSR write; words = the lists section copied to an aligned
// buffer (word 0 at byte links_begin); *first = min(list byte * 2 + kind).
cudaError_t ingest_links(const uint32_t* words, const uint64_t* node_off, uint64_t links_begin, const uint8_t* levels,
                         uint32_t n, uint32_t m0p, uint32_t mp, const uint32_t* up_off, uint32_t* adj0,
                         uint32_t* adjU, unsigned long long* first, cudaStream_t stream);
cudaError_t ingest_dead(const uint8_t* flags, uint32_t n, uint32_t* dead, unsigned long long* dead_count,
                        cudaStream_t stream);
// flags_out[0] counts live keys equal to ~0, [1] is set on a repeated live
// key, [2] when some key differs from its node id.
cudaError_t ingest_live_keys(const uint64_t* keys, const uint8_t* flags, uint32_t n, unsigned long long* table,
                             uint64_t cap, unsigned int* flags_out, cudaStream_t stream);

// Derives int8 codes and their squared norms from offsets and scale
// (ScalarQuantizer::encode_into, src/quantization.rs:73-81).
cudaError_t launch_encode_codes(const float* vec, uint32_t n, uint32_t dim, uint32_t dp, uint32_t dc,
                                const float* offset, float scale, int8_t* codes, int32_t* norms,
                                cudaStream_t stream);

// Exact FP32 brute force in the reference kernel order (K1 per row) with a
// per-query top-k merge.
struct BruteArgs {
    const float* base = nullptr;  // n * dp, prepared
    const uint64_t* keys = nullptr;
    uint32_t n = 0, dim = 0, dp = 0;
    int metric = 0;
    const float* queries = nullptr;  // nq * dim raw
    uint32_t nq = 0, k = 10;
    uint64_t* out_keys = nullptr;
    float* out_dist = nullptr;
    uint32_t* out_count = nullptr;
    int32_t* out_status = nullptr;
    // scratch
    float* qprep = nullptr;         // nq * dp
    uint64_t* part = nullptr;       // nq * tiles * k partial top-k (packed dist key, row)
    uint32_t tiles = 0;
    // Optional filter (BruteForceIndex::search_filtered): a row is scored
    // only when its bit is set; bit = key, or row index with filter_by_row.
    // Query q uses bitmap filter_ids[q] (or q) at filter_stride words each
    // (stride 0: one shared bitmap), unless filter_used[q] == 0.
    const uint64_t* filter_bits = nullptr;
    uint64_t filter_nbits = 0;
    uint64_t filter_stride = 0;
    const uint8_t* filter_used = nullptr;
    const uint32_t* filter_ids = nullptr;
    int filter_by_row = 0;
};
cudaError_t launch_brute_fp32(const BruteArgs& a, cudaStream_t stream);
// Query preparation only (vector::check, cosine normalisation) into a.qprep.
cudaError_t launch_brute_prep(const BruteArgs& a, cudaStream_t stream);
// Exact FP32 re-rank of packed (approx distance bits << 32 | row) candidates
// whose approximate distance is <= thr2[q]; writes a.out_* (status 25 when a
// query's candidate list overflowed).
cudaError_t launch_brute_rerank(const BruteArgs& a, const uint64_t* cand, const uint32_t* cand_count, uint32_t cand_cap,
                                const float* thr2, cudaStream_t stream);

// Fixed device scratch of the allocation-free brute-force entry point.
constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;  // 8 MiB per device
constexpr int kMaxDevices = 64;
// Device address of that scratch on the current device (looked up once per
// device with cudaGetSymbolAddress, then cached).
cudaError_t noalloc_scratch_address(void** out);
// Splits the scratch into prepared queries and per-slice top-k lists for a
// batch; false when even one slice does not fit.
bool noalloc_layout(uint32_t nq, uint32_t dp, uint32_t kk, uint32_t want_slices, size_t* qprep_bytes,
                    uint32_t* slices);

}  // namespace hnswgpu
