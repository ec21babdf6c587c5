// C ABI: the drop-in boundary (include/hnsw_gpu.h).
//
// Host-side work here is plumbing: validating the file (host loader),
// flattening the graph into the device layout, staging buffers, choosing a
// scratch geometry per call and launching the kernels. No search result is
// ever computed on the host.
#include "hnsw_gpu.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <functional>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "capi_internal.hpp"
#include "gpu_build.hpp"

using namespace hnswgpu;

namespace hnswgpu {

namespace {
thread_local std::string g_last_error;

std::string format_error_message(const Err& e) {
    char buf[256];
    switch (e.status) {
        case HNSW_ERR_FORMAT_BAD_MAGIC: return "invalid index file: missing HNSWIDX magic bytes";
        case HNSW_ERR_FORMAT_UNSUPPORTED_VERSION:
            std::snprintf(buf, sizeof buf, "invalid index file: unsupported format version %llu", (unsigned long long)e.a);
            return buf;
        case HNSW_ERR_FORMAT_TRUNCATED: return "invalid index file: unexpected end of input";
        case HNSW_ERR_FORMAT_CHECKSUM:
            std::snprintf(buf, sizeof buf, "invalid index file: checksum mismatch: stored %#010llx, computed %#010llx",
                          (unsigned long long)e.a, (unsigned long long)e.b);
            return buf;
        case HNSW_ERR_FORMAT_TRAILING_BYTES: return "invalid index file: unexpected bytes after the last section";
        case HNSW_ERR_FORMAT_INVALID: return "invalid index file: invalid field: " + e.what;
        case HNSW_ERR_MEMORY_LIMIT_EXCEEDED:
            std::snprintf(buf, sizeof buf,
                          "loading the index needs %llu bytes of memory, more than the limit of %llu",
                          (unsigned long long)e.a, (unsigned long long)e.b);
            return buf;
        case HNSW_ERR_DUPLICATE_KEY:
            std::snprintf(buf, sizeof buf, "key %llu is already present", (unsigned long long)e.a);
            return buf;
        case HNSW_ERR_NON_FINITE_VECTOR: return "vector contains NaN or infinite values";
        case HNSW_ERR_ZERO_VECTOR: return "zero vector has no direction under cosine distance";
        case HNSW_ERR_CAPACITY_EXCEEDED: return "index capacity exceeded";
        case HNSW_ERR_DIMENSION_MISMATCH: return "dimension mismatch";
        default: return e.what;
    }
}

}  // namespace

const char* last_error_text() { return g_last_error.c_str(); }

int set_error(int status, const std::string& msg) {
    g_last_error = msg;
    return status;
}

int from_err(const Err& e) { return e ? set_error(e.status, format_error_message(e)) : HNSW_OK; }

int cuda_fail(cudaError_t e, const char* where) {
    if (e == cudaErrorMemoryAllocation)
        return set_error(HNSW_ERR_OUT_OF_DEVICE_MEMORY, std::string(where) + ": " + cudaGetErrorString(e));
    return set_error(HNSW_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

// Persistent warps spill to global memory instead of restarting, so their
// visited hash is sized near the typical visit count (about 12 per unit of
// ef on the 1M x 128 workload, p99 about 25); plain warps size it for the tail.
SearchGeometry pick_geometry(uint32_t ef_max, uint32_t dp, uint32_t dc, bool persistent, bool filtered, uint32_t n) {
    constexpr uint32_t kSmemBudget = 220 * 1024;
    const int tags = g_visit_tag_bits.load();
    SearchGeometry g;
    g.ef_cap = std::min<uint32_t>(1024, std::max<uint32_t>(32, round_up(ef_max, 32)));
    g.cand_cap = 2 * g.ef_cap + 32;
    uint32_t want = g.ef_cap * (persistent ? 32 : 48);
    uint32_t h = 2048;
    while (h < want && h < 32768) h <<= 1;
    g.hash_cap = h;
    // A persistent hash of 16-bit tags gets twice the slots for the bytes of
    // 32-bit ids, up to 8192 slots (fewer spills; measured on the 1M x 128
    // workload: ef = 64 2.35 ms with 4096 slots against 3.64 ms with 2048;
    // at ef = 256 a 16384-slot hash costs more residency than it saves).
    if (persistent && 2 * h <= 8192) {
        SearchGeometry t = g;
        t.hash_cap = 2 * h;
        set_hash_tags(t, n, tags);
        if (t.tag16) g.hash_cap = 2 * h;
    }
    // The sizing rules below count 32-bit slots (measured: they pick 4096
    // slots at ef = 64 and 8192 at ef = 256 for plain warps, the fastest
    // sizes with tags as well).
    while (geometry_bytes_per_warp(g, dp, dc) > kSmemBudget && g.hash_cap > 1024) g.hash_cap >>= 1;
    // Keep at least four warps per SM: a query that outgrows a smaller hash
    // continues in its spill bitmap (persistent) or the retry pass (plain),
    // which costs less than idle SMs (measured: a 64 KB hash at ef = 512 left
    // two warps per SM).
    while (geometry_bytes_per_warp(g, dp, dc) > kSmemBudget / 4 && g.hash_cap > 4096) g.hash_cap >>= 1;
    set_hash_tags(g, n, tags);
    // Warps per block that maximise resident warps per SM, the fewest on a
    // tie (a plain block holds its SM slot until its slowest query ends).
    uint32_t best_warps = 0, best_wpb = 1;
    for (uint32_t wpb : {1u, 2u, 4u, 8u}) {
        SearchGeometry t = g;
        t.warps_per_block = wpb;
        if (size_t(geometry_bytes_per_warp(t, dp, dc)) * wpb > kSmemBudget) continue;
        uint32_t warps = 0;
        if (persistent_warps(t, dp, dc, 1, &warps) != cudaSuccess) continue;
        if (warps > best_warps) {
            best_warps = warps;
            best_wpb = wpb;
        }
    }
    g.warps_per_block = best_wpb;
    // Filtered batches: admitted results fill slowly, so queues grow long;
    // the cold-list variant keeps them in the fast kernel.
    g.cold = persistent && filtered ? 1 : 0;
    return g;
}

}  // namespace hnswgpu

// Ensures the retry workspaces of a slot (visited bitmap over all nodes, heaps).
static int ensure_retry(hnsw_gpu_index* gi, Slot* s, uint32_t ef_cap) {
    const uint32_t warps = uint32_t(gi->num_sms) * 4;
    const uint32_t cand_cap = std::max<uint32_t>(1u << 14, 4 * ef_cap);
    const uint64_t words = (uint64_t(gi->view.n) + 31) / 32 + 1;
    CU(s->g_results.ensure(size_t(warps) * (ef_cap + 1) * 8), "cudaMalloc retry results");
    CU(s->g_cands.ensure(size_t(warps) * (cand_cap + 1) * 8), "cudaMalloc retry candidates");
    CU(s->g_visited.ensure(size_t(warps) * words * 4), "cudaMalloc retry visited");
    s->g_warps = warps;
    s->g_ef_cap = ef_cap;
    s->g_cand_cap = cand_cap;
    s->g_words = words;
    return HNSW_OK;
}

// Enqueues one search on `stream` with device pointers. ef_max bounds every
// per-query max(ef, k) of the batch.
// The schedule comes from, in order: `force` (the autotuner's trials), the
// fixed schedule, the tuning table, the occupancy heuristic. HNSW_MODE_AUTO
// resolves to the tuned mode of the bucket, else persistent.
// Builds the tensor-core traversal rows on first use (and the low parts on
// the first BF16X3 search). The build is waited for before the lock is
// released, so a search on any stream that finds them ready can read them.
static int ensure_tc_rows(hnsw_gpu_index* gi, bool lo, cudaStream_t stream) {
    std::lock_guard<std::mutex> l(gi->tc_mu);
    if (gi->tc_hi_ready && (!lo || gi->tc_lo_ready)) return HNSW_OK;
    const DeviceIndexView& v = gi->view;
    const uint32_t dt = round_up(v.dim, 32);
    const size_t row_bytes = size_t(v.n) * dt * 2;
    CU(gi->tc_hi.ensure(std::max<size_t>(row_bytes, 16)), "cudaMalloc tensor-core rows");
    if (lo) CU(gi->tc_lo.ensure(std::max<size_t>(row_bytes, 16)), "cudaMalloc tensor-core low parts");
    if (v.metric == HNSW_METRIC_L2) CU(gi->tc_norm.ensure(std::max<size_t>(size_t(v.n) * 4, 4)), "cudaMalloc row norms");
    CU(launch_tc_rows(v.vec, v.n, v.dim, v.dp, dt, gi->tc_hi.as<uint4>(), lo ? gi->tc_lo.as<uint4>() : nullptr,
                      v.metric == HNSW_METRIC_L2 ? gi->tc_norm.as<float>() : nullptr, stream),
       "tensor-core rows");
    CU(cudaStreamSynchronize(stream), "tensor-core rows");
    gi->tc_hi_ready = true;
    if (lo) gi->tc_lo_ready = true;
    return HNSW_OK;
}

int hnswgpu::enqueue_search(hnsw_gpu_index* gi, Slot* s, const float* d_q, size_t nq, const hnsw_search_opts& o_in,
                          const uint32_t* d_ks, const uint32_t* d_efs, const uint64_t* d_fbits, const uint8_t* d_fused,
                          const uint32_t* d_fids,
                          uint64_t* d_keys, float* d_dist, uint32_t* d_count, int32_t* d_status, uint32_t ef_max,
                          uint32_t out_stride, cudaStream_t stream, const SearchGeometry* force, bool publish) {
    hnsw_search_opts o = o_in;
    if (o.mode != HNSW_MODE_PLAIN && o.mode != HNSW_MODE_PERSISTENT && o.mode != HNSW_MODE_AUTO)
        return set_error(HNSW_ERR_INVALID_ARGUMENT, "unknown search mode");
    if (o.traversal < HNSW_TRAVERSAL_F32 || o.traversal > HNSW_TRAVERSAL_BF16X3)
        return set_error(HNSW_ERR_INVALID_ARGUMENT, "unknown traversal");
    if (o.traversal && o.quantized)
        return set_error(HNSW_ERR_INVALID_ARGUMENT, "the tensor-core traversal does not combine with quantized search");
    if (o.traversal) {
        const int r = ensure_tc_rows(gi, o.traversal == HNSW_TRAVERSAL_BF16X3, stream);
        if (r != HNSW_OK) return r;
    }
    const uint32_t tcb = o.traversal ? round_up(gi->view.dim, 32) * 2u * (o.traversal == HNSW_TRAVERSAL_BF16X3 ? 2u : 1u)
                                     : 0u;
    SearchGeometry geo{0, 0, 0, 0, 0};
    if (force) {
        geo = *force;
    } else if (gi->fixed.ef_cap) {
        geo = gi->fixed;
    } else {
        std::lock_guard<std::mutex> l(gi->tune_mu);
        const hnsw_gpu_index::Tuned& t = gi->tuned[tune_bucket(ef_max)];
        if (o.mode == HNSW_MODE_AUTO) o.mode = t.mode >= 0 ? t.mode : HNSW_MODE_PERSISTENT;
        if (t.geo[o.mode].ef_cap) geo = t.geo[o.mode];
    }
    if (o.mode == HNSW_MODE_AUTO) o.mode = HNSW_MODE_PERSISTENT;
    const bool persistent = o.mode == HNSW_MODE_PERSISTENT, filtered = d_fbits != nullptr;
    if (!geo.ef_cap) geo = pick_geometry(ef_max, gi->view.dp, gi->view.dc, persistent, filtered, gi->view.n);
    geo.stage_row_bytes =
        geo.stage_rows ? ((o.quantized && gi->view.quantized) ? gi->view.dc : gi->view.dp * 4) : 0;
    geo.tc_bytes = tcb;
    const int tags = g_visit_tag_bits.load();
    set_hash_tags(geo, gi->view.n, tags);
    // A schedule tuned on int8 rows may not fit f32 rows (or the tensor-core
    // query operands): the heuristic's, with the visited hash halved until
    // it fits.
    if (size_t(geometry_bytes_per_warp(geo, gi->view.dp, gi->view.dc)) * geo.warps_per_block > 220 * 1024) {
        geo = pick_geometry(ef_max, gi->view.dp, gi->view.dc, persistent, filtered, gi->view.n);
        geo.tc_bytes = tcb;
        set_hash_tags(geo, gi->view.n, tags);
        while (size_t(geometry_bytes_per_warp(geo, gi->view.dp, gi->view.dc)) * geo.warps_per_block > 220 * 1024 &&
               geo.hash_cap > 1024) {
            geo.hash_cap >>= 1;
            set_hash_tags(geo, gi->view.n, tags);
        }
    }
    if (!persistent) geo.cold = 0;  // cold lists need the persistent warps' chunk tables
    // work: [0] next query, [1] overflow count, [2] [3] cold chunks handed
    // out by the fast (cold variant) and retry kernels, [4] last-resort count.
    CU(s->work.ensure(32), "cudaMalloc work counters");
    CU(s->overflow.ensure(std::max<size_t>(nq, 1) * 4), "cudaMalloc overflow list");
    CU(s->overflow2.ensure(std::max<size_t>(nq, 1) * 4), "cudaMalloc overflow list");
    CU(cudaMemsetAsync(s->work.p, 0, 32, stream), "memset work counters");
    int r = ensure_retry(gi, s, std::max(geo.ef_cap, round_up(ef_max, 32)));
    if (r != HNSW_OK) return r;
    SearchArgs a;
    a.ix = gi->view;
    a.queries = d_q;
    a.nq = uint32_t(nq);
    a.k = o.k;
    a.ef = o.ef;
    a.ks = d_ks;
    a.efs = d_efs;
    a.quantized = o.quantized;
    a.traversal = o.traversal;
    if (o.traversal) {
        a.ix.tc_hi = gi->tc_hi.as<uint4>();
        a.ix.tc_lo = o.traversal == HNSW_TRAVERSAL_BF16X3 ? gi->tc_lo.as<uint4>() : nullptr;
        a.ix.xnorm = gi->view.metric == HNSW_METRIC_L2 ? gi->tc_norm.as<float>() : nullptr;
        a.ix.dt = round_up(gi->view.dim, 32);
    }
    a.filter_bits = d_fbits;
    a.filter_nbits = o.filter_nbits;
    a.filter_stride = o.filter_stride;
    a.filter_used = d_fused;
    a.filter_ids = d_fids;
    a.filter_by_node = o.filter_by_node;
    a.out_keys = d_keys;
    a.out_dist = d_dist;
    a.out_count = d_count;
    a.out_status = d_status;
    a.out_stride = out_stride;
    a.publish = publish ? 1 : 0;
#ifdef HNSW_DEVICE_CHECKS
    if (!gi->chk.p) {
        CU(gi->chk.ensure(16), "cudaMalloc check word");
        CU(cudaMemset(gi->chk.p, 0, 16), "clear check word");
    }
    a.chk = gi->chk.as<uint32_t>();
#endif
    if (gi->counters) {
        CU(s->counters.ensure(std::max<size_t>(nq, 1) * 16), "cudaMalloc counters");
        a.counters = s->counters.as<uint32_t>();
    }
    a.work_next = s->work.as<uint32_t>();
    a.overflow_count = s->work.as<uint32_t>() + 1;
    a.overflow_list = s->overflow.as<uint32_t>();
    a.persistent = o.mode == HNSW_MODE_PERSISTENT ? 1 : 0;
    if (a.persistent) {
        uint32_t warps = 0;
        CU(persistent_warps(geo, gi->view.dp, gi->view.dc, gi->num_sms, &warps), "occupancy");
        const uint32_t words = ((gi->view.n + 31) / 32 + 3) & ~3u;
        const uint32_t cand_cap = std::max<uint32_t>(8192, 4 * geo.ef_cap);
        const size_t bits_bytes = size_t(warps) * words * 4;
        if (bits_bytes > s->spill_bits.bytes) {
            CU(s->spill_bits.ensure(bits_bytes), "cudaMalloc spill bitmaps");
            CU(cudaMemsetAsync(s->spill_bits.p, 0, s->spill_bits.bytes, stream), "memset spill bitmaps");
        }
        if (!geo.cold) {
            CU(s->spill_cands.ensure(size_t(warps) * (cand_cap + 1) * 8), "cudaMalloc spill candidates");
            a.spill_cands = s->spill_cands.as<uint64_t>();
            a.spill_cand_cap = cand_cap;
        }
        a.spill_bits = s->spill_bits.as<uint32_t>();
        a.spill_words = words;
        a.spill_slots = warps;
    }
    // Cold candidate lists (the cold variant's persistent warps, then the
    // retry warps, which reuse the whole pool): 8 entries per node or 32
    // chunks (32768 candidates) per warp, whichever is more, 2 GiB at most. A
    // list never holds more entries than there are nodes; a query whose warp
    // finds the pool empty moves on to the next pass.
    const uint32_t tab_cap = (gi->view.n + kColdChunk - 1) / kColdChunk + 2;
    {
        const uint32_t slots = geo.cold ? std::max(a.spill_slots, s->g_warps) : s->g_warps;
        const uint64_t want = std::max<uint64_t>((uint64_t(gi->view.n) * 8 + kColdChunk - 1) / kColdChunk,
                                                 uint64_t(slots) * 32);
        const uint32_t chunks = geo.cold_chunks ? geo.cold_chunks : uint32_t(std::min<uint64_t>(want, 1u << 18));
        CU(s->cold_pool.ensure(size_t(chunks) * kColdChunk * 8), "cudaMalloc cold candidate pool");
        CU(s->cold_tab.ensure(size_t(slots) * tab_cap * 4), "cudaMalloc cold chunk tables");
        a.cold_pool = s->cold_pool.as<uint64_t>();
        a.cold_chunks = chunks;
        a.cold_next = s->work.as<uint32_t>() + 2;
        a.cold_tab = s->cold_tab.as<uint32_t>();
        a.cold_tab_cap = tab_cap;
        a.cold_slots = slots;
    }
    a.g_results = s->g_results.as<uint64_t>();
    a.g_cands = s->g_cands.as<uint64_t>();
    a.g_visited = s->g_visited.as<uint32_t>();
    a.g_ef_cap = s->g_ef_cap;
    a.g_cand_cap = s->g_cand_cap;
    a.g_visited_words = s->g_words;
    // Last-resort regions: kLastResortWarps rows of tab_cap chunks each,
    // chunk table rows preassigned once.
    if (s->last_tab.bytes < size_t(kLastResortWarps) * tab_cap * 4) {
        CU(s->last_pool.ensure(size_t(kLastResortWarps) * tab_cap * kColdChunk * 8), "cudaMalloc last-resort pool");
        CU(s->last_tab.ensure(size_t(kLastResortWarps) * tab_cap * 4), "cudaMalloc last-resort table");
        std::vector<uint32_t> ids(size_t(kLastResortWarps) * tab_cap);
        for (size_t i = 0; i < ids.size(); ++i) ids[i] = uint32_t(i);
        CU(cudaMemcpy(s->last_tab.p, ids.data(), ids.size() * 4, cudaMemcpyHostToDevice), "copy last-resort table");
    }
    a.overflow_list2 = s->overflow2.as<uint32_t>();
    a.overflow_count2 = s->work.as<uint32_t>() + 4;
    if (o.exact_below > 0.0f && d_fbits) {
        CU(s->planned.ensure(std::max<size_t>(nq, 1)), "cudaMalloc planner flags");
        a.plan_max = uint32_t(std::max(1.0, std::floor(double(o.exact_below) * double(gi->view.live))));
        CU(launch_plan(a, s->planned.as<uint8_t>(), stream), "planner kernel");
        a.planned = s->planned.as<uint8_t>();
    }
    CU(launch_search(a, geo, gi->num_sms, stream), "search kernel");
    CU(launch_search_retry(a, s->g_warps, stream), "search retry kernel");
    SearchArgs last = a;
    last.overflow_list = a.overflow_list2;
    last.overflow_count = a.overflow_count2;
    last.overflow_list2 = nullptr;
    last.overflow_count2 = nullptr;
    last.cold_pool = s->last_pool.as<uint64_t>();
    last.cold_chunks = kLastResortWarps * tab_cap;
    last.cold_next = nullptr;
    last.cold_tab = s->last_tab.as<uint32_t>();
    last.cold_tab_cap = tab_cap;
    last.cold_slots = kLastResortWarps;
    last.cold_private = 1;
    CU(launch_search_retry(last, kLastResortWarps, stream), "search last-resort kernel");
    return HNSW_OK;
}

extern "C" {

const char* hnsw_last_error(void) { return hnswgpu::last_error_text(); }

uint32_t hnsw_crc32(const uint8_t* bytes, size_t len) { return crc32(bytes, len); }

static void fill_info(const HostIndex& ix, uint64_t required, hnsw_index_info* out) {
    std::memset(out, 0, sizeof *out);
    out->dim = ix.dim;
    out->metric = uint32_t(ix.metric);
    out->m = ix.params.m;
    out->m0 = ix.params.m0;
    out->ef_construction = ix.params.ef_construction;
    out->quantized = ix.quantized ? 1 : 0;
    out->nodes = uint32_t(ix.node_count());
    out->live = uint32_t(ix.key_to_id.size());
    out->top_level = ix.has_entry() ? ix.top_level() : 0;
    out->entry = ix.has_entry() ? ix.entry_id() : kSentinel;
    out->seed = ix.params.seed;
    out->level_multiplier = ix.params.level_multiplier;
    out->required_memory = required;
}

int hnsw_validate_bytes(const uint8_t* bytes, size_t len, uint64_t max_memory, hnsw_index_info* info) {
    if (!bytes && len) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null buffer");
    static const uint8_t empty = 0;
    HostIndex ix;
    uint64_t required = 0;
    Err e = load_index(bytes ? bytes : &empty, len, max_memory, &ix, &required);
    if (e) return from_err(e);
    if (info) fill_info(ix, required, info);
    return HNSW_OK;
}

// Device ingest (ingest.cu): every check of io::read in the reference's
// order, the per-byte and per-node ones on the device, building the device
// layout from one copy of the file. Temporaries are freed on every path.
static int ingest_open(hnsw_gpu_index* gi, const uint8_t* bytes, size_t len, uint64_t max_memory) {
    size_t body_len = 0;
    uint32_t stored = 0;
    Err e = check_envelope(bytes, len, &body_len, &stored);
    if (e) return from_err(e);
    struct Tmp {
        DBuf file, part, pow8, word, words, noff, upoff_tmp, table, flags;
        ~Tmp() {
            for (DBuf* b : {&file, &part, &pow8, &word, &words, &noff, &upoff_tmp, &table, &flags}) b->release();
        }
    } t;
    cudaStream_t st = nullptr;
    // 1. The file on the device; CRC-32 of the body (verify_envelope).
    CU(t.file.ensure(std::max<size_t>(len, 16)), "cudaMalloc file");
    CU(cudaMemcpy(t.file.p, bytes, len, cudaMemcpyHostToDevice), "copy file");
    const uint8_t* df = t.file.as<uint8_t>();
    const size_t nchunks = std::max<size_t>(1, (body_len + kIngestCrcChunk - 1) / kIngestCrcChunk);
    CU(t.part.ensure(nchunks * 4), "cudaMalloc crc chunks");
    CU(t.pow8.ensure(64 * 4), "cudaMalloc crc powers");
    CU(t.word.ensure(64), "cudaMalloc crc word");
    uint32_t computed = 0;
    CU(ingest_crc(df, body_len, t.part.as<uint32_t>(), t.pow8.as<uint32_t>(), t.word.as<uint32_t>(), &computed, st),
       "crc kernel");
    if (computed != stored) return from_err(checksum_error(stored, computed));
    // 2. Header, columns, list counts, memory limit (host).
    FileLayout L;
    e = scan_layout(bytes, body_len, max_memory, &L);
    if (e) return from_err(e);
    const uint32_t n = L.n;
    const size_t nn = std::max<size_t>(n, 1);
    DeviceIndexView& v = gi->view;
    v.n = n;
    v.dim = L.dim;
    v.dp = round_up(L.dim, 32);
    v.dc = round_up(L.dim, 16);
    v.m = L.params.m;
    v.m0 = L.params.m0;
    v.mp = round_up(L.params.m, 32);
    v.m0p = round_up(L.params.m0, 32);
    v.metric = L.metric;
    v.quantized = L.quantized ? 1 : 0;
    // 3. Vectors into padded rows, then read_nodes' checks (device).
    CU(t.flags.ensure(64), "cudaMalloc flags");
    unsigned long long* first = t.flags.as<unsigned long long>();
    CU(cudaMemset(t.flags.p, 0xFF, 8), "memset flags");
    CU(gi->vec.ensure(nn * v.dp * 4), "cudaMalloc vectors");
    if (v.dp != v.dim) CU(cudaMemset(gi->vec.p, 0, nn * v.dp * 4), "memset vectors");
    if (n)
        CU(cudaMemcpy2D(gi->vec.p, size_t(v.dp) * 4, df + (L.vectors - bytes), size_t(v.dim) * 4, size_t(v.dim) * 4, n,
                        cudaMemcpyDeviceToDevice),
           "copy vectors");
    v.vec = gi->vec.as<float>();
    CU(ingest_check_vectors(v.vec, n, v.dim, v.dp, L.metric == HNSW_METRIC_COSINE, first, st), "vector checks");
    unsigned long long bad = 0;
    CU(cudaMemcpy(&bad, first, 8, cudaMemcpyDeviceToHost), "vector checks");
    if (bad != ~0ull)
        return from_err(invalid_field((bad & 1ull) ? "cosine vector is not unit length" : "vector out of range"));
    // 4. read_links' checks and the CSR (device).
    std::vector<uint32_t> off(nn, 0);
    size_t blocks = 0;
    for (uint32_t id = 0; id < n; ++id) {
        off[id] = uint32_t(blocks);
        blocks += L.levels[id];
    }
    CU(gi->adj0.ensure(nn * v.m0p * 4), "cudaMalloc adj0");
    CU(cudaMemset(gi->adj0.p, 0xFF, nn * v.m0p * 4), "memset adj0");
    CU(gi->upoff.ensure(nn * 4), "cudaMalloc up_off");
    CU(cudaMemcpy(gi->upoff.p, off.data(), nn * 4, cudaMemcpyHostToDevice), "copy up_off");
    CU(gi->adjU.ensure(std::max<size_t>(blocks, 1) * v.mp * 4), "cudaMalloc adjU");
    CU(cudaMemset(gi->adjU.p, 0xFF, std::max<size_t>(blocks, 1) * v.mp * 4), "memset adjU");
    v.adj0 = gi->adj0.as<uint32_t>();
    v.up_off = gi->upoff.as<uint32_t>();
    v.adjU = gi->adjU.as<uint32_t>();
    const size_t link_bytes = L.links_end - L.links_begin;
    CU(t.words.ensure(std::max<size_t>(link_bytes, 16)), "cudaMalloc lists");
    if (link_bytes) CU(cudaMemcpy(t.words.p, df + L.links_begin, link_bytes, cudaMemcpyDeviceToDevice), "copy lists");
    CU(t.noff.ensure(nn * 8), "cudaMalloc list offsets");
    if (n) CU(cudaMemcpy(t.noff.p, L.node_off.data(), size_t(n) * 8, cudaMemcpyHostToDevice), "copy list offsets");
    CU(cudaMemset(t.flags.p, 0xFF, 8), "memset flags");
    CU(ingest_links(t.words.as<uint32_t>(), t.noff.as<uint64_t>(), L.links_begin, df + (L.levels - bytes), n, v.m0p,
                    v.mp, gi->upoff.as<uint32_t>(), gi->adj0.as<uint32_t>(), gi->adjU.as<uint32_t>(), first, st),
       "list checks");
    CU(cudaMemcpy(&bad, first, 8, cudaMemcpyDeviceToHost), "list checks");
    if (bad != ~0ull) return from_err(invalid_field((bad & 1ull) ? "duplicate neighbor id" : "neighbor id"));
    // 5. Quantizer section and trailing bytes (host).
    std::vector<float> q_offset;
    float q_scale = 0.0f;
    e = scan_tail(bytes, L, &q_offset, &q_scale);
    if (e) return from_err(e);
    v.scale = q_scale;
    // 6. Keys: distinct among live nodes (device), then the entry point.
    CU(gi->keys.ensure(nn * 8), "cudaMalloc keys");
    if (n) CU(cudaMemcpy(gi->keys.p, df + (L.keys - bytes), size_t(n) * 8, cudaMemcpyDeviceToDevice), "copy keys");
    v.keys = gi->keys.as<uint64_t>();
    uint64_t cap = 2;
    while (cap < 2 * uint64_t(nn)) cap <<= 1;
    CU(t.table.ensure(cap * 8), "cudaMalloc key set");
    CU(cudaMemset(t.table.p, 0xFF, cap * 8), "memset key set");
    unsigned int* kflags = reinterpret_cast<unsigned int*>(t.flags.as<uint8_t>() + 16);
    CU(cudaMemset(kflags, 0, 12), "memset key flags");
    CU(ingest_live_keys(v.keys, df + (L.dead - bytes), n, t.table.as<unsigned long long>(), cap, kflags, st),
       "key checks");
    unsigned int kf[3] = {0, 0, 0};
    CU(cudaMemcpy(kf, kflags, 12, cudaMemcpyDeviceToHost), "key checks");
    if (kf[1]) return from_err(invalid_field("duplicate live key"));
    v.keys_are_ids = kf[2] ? 0 : 1;
    uint64_t entry_word = 0;
    e = check_entry(L, &entry_word);
    if (e) return from_err(e);
    v.entry = n ? uint32_t(entry_word) : kSentinel;
    v.top = n ? uint32_t(entry_word >> 32) : 0;
    // 7. Tombstones.
    CU(gi->dead.ensure(((nn + 31) / 32) * 4), "cudaMalloc dead");
    CU(cudaMemset(gi->dead.p, 0, ((nn + 31) / 32) * 4), "memset dead");
    unsigned long long* dead_count = first;
    CU(cudaMemset(dead_count, 0, 8), "memset dead count");
    CU(ingest_dead(df + (L.dead - bytes), n, gi->dead.as<uint32_t>(), dead_count, st), "tombstones");
    unsigned long long ndead = 0;
    CU(cudaMemcpy(&ndead, dead_count, 8, cudaMemcpyDeviceToHost), "tombstones");
    v.dead = gi->dead.as<uint32_t>();
    v.has_dead = ndead ? 1 : 0;
    v.live = uint32_t(n - ndead);
    // 8. Quantizer: offsets, then codes derived on the device.
    if (L.quantized) {
        std::vector<float> offp(v.dp, 0.0f);
        std::copy(q_offset.begin(), q_offset.end(), offp.begin());
        CU(gi->offset.ensure(offp.size() * 4), "cudaMalloc offsets");
        CU(cudaMemcpy(gi->offset.p, offp.data(), offp.size() * 4, cudaMemcpyHostToDevice), "copy offsets");
        CU(gi->codes.ensure(nn * v.dc), "cudaMalloc codes");
        CU(gi->norms.ensure(nn * 4), "cudaMalloc code norms");
        CU(launch_encode_codes(v.vec, n, v.dim, v.dp, v.dc, gi->offset.as<float>(), v.scale, gi->codes.as<int8_t>(),
                               gi->norms.as<int32_t>(), st),
           "encode codes");
        v.q_offset = gi->offset.as<float>();
        v.codes = gi->codes.as<int8_t>();
        v.code_norm = gi->norms.as<int32_t>();
    }
    CU(cudaDeviceSynchronize(), "ingest");
    hnsw_index_info& info = gi->info;
    std::memset(&info, 0, sizeof info);
    info.dim = L.dim;
    info.metric = L.metric;
    info.m = L.params.m;
    info.m0 = L.params.m0;
    info.ef_construction = L.params.ef_construction;
    info.quantized = L.quantized ? 1 : 0;
    info.nodes = n;
    info.live = v.live;
    info.top_level = v.top;
    info.entry = v.entry;
    info.seed = L.params.seed;
    info.level_multiplier = L.params.level_multiplier;
    info.required_memory = L.required;
    info.device_bytes = gi->vec.bytes + gi->adj0.bytes + gi->upoff.bytes + gi->adjU.bytes + gi->keys.bytes +
                        gi->dead.bytes + gi->offset.bytes + gi->codes.bytes + gi->norms.bytes;
    return HNSW_OK;
}

int hnsw_gpu_index_open(const uint8_t* bytes, size_t len, uint64_t max_memory, int device, hnsw_gpu_index** out) {
    if (!out) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null output handle");
    *out = nullptr;
    if (!bytes && len) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null buffer");
    static const uint8_t empty = 0;
    int ndev = 0;
    cudaError_t ce = cudaGetDeviceCount(&ndev);
    if (ce != cudaSuccess || ndev == 0)
        return set_error(HNSW_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(ce));
    if (device < 0 || device >= ndev) return set_error(HNSW_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    DeviceGuard dg(device);
    TraceRange trace("hnsw.index_open");
    std::unique_ptr<hnsw_gpu_index> gi(new hnsw_gpu_index());
    gi->device = device;
    gi->slots.device = device;
    cudaDeviceGetAttribute(&gi->num_sms, cudaDevAttrMultiProcessorCount, device);
    int s = ingest_open(gi.get(), bytes ? bytes : &empty, len, max_memory);
    if (s != HNSW_OK) return s;
    if (gi->view.dim > 8192) return set_error(HNSW_ERR_INVALID_ARGUMENT, "dimension above the device path's limit of 8192");
    *out = gi.release();
    return HNSW_OK;
}

void hnsw_gpu_index_close(hnsw_gpu_index* index) { delete index; }

int hnsw_gpu_index_info(const hnsw_gpu_index* index, hnsw_index_info* out) {
    if (!index || !out) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    *out = index->info;
    return HNSW_OK;
}

int hnsw_gpu_set_tombstones(hnsw_gpu_index* index, const uint8_t* deleted, size_t nodes) {
    if (!index || (!deleted && nodes)) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    if (nodes != index->view.n) return set_error(HNSW_ERR_DIMENSION_MISMATCH, "tombstone column length != node count");
    DeviceGuard dg(index->device);
    std::vector<uint32_t> dead((std::max<size_t>(nodes, 1) + 31) / 32, 0);
    uint32_t live = 0;
    for (size_t id = 0; id < nodes; ++id) {
        if (deleted[id] > 1) return set_error(HNSW_ERR_INVALID_ARGUMENT, "tombstone flags must be 0 or 1");
        if (deleted[id]) dead[id >> 5] |= 1u << (id & 31);
        else ++live;
    }
    CU(cudaMemcpy(index->dead.p, dead.data(), dead.size() * 4, cudaMemcpyHostToDevice), "copy tombstones");
    index->view.live = live;
    index->view.has_dead = live != nodes ? 1 : 0;
    index->info.live = live;
    return HNSW_OK;
}

int hnsw_gpu_set_schedule(hnsw_gpu_index* index, const hnsw_schedule* sc) {
    if (!index) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null index");
    if (!sc) {
        index->fixed = SearchGeometry{0, 0, 0, 0, 0};
        return HNSW_OK;
    }
    const bool hash_ok = sc->hash_cap >= 64 && sc->hash_cap % 64 == 0 && sc->hash_cap <= (1u << 20);
    if (sc->ef_cap < 32 || sc->ef_cap > 1024 || sc->ef_cap % 32 || sc->cand_cap < sc->ef_cap || !hash_ok ||
        sc->warps_per_block < 1 || sc->warps_per_block > 8 || sc->stage_rows > 32)
        return set_error(HNSW_ERR_INVALID_ARGUMENT, "schedule out of range");
    SearchGeometry g;
    g.ef_cap = sc->ef_cap;
    g.cand_cap = sc->cand_cap;
    g.hash_cap = sc->hash_cap;
    g.warps_per_block = sc->warps_per_block;
    g.cold_chunks = sc->cold_chunks;
    g.stage_rows = sc->stage_rows;
    g.cold = sc->cold ? 1 : 0;
    if (size_t(geometry_bytes_per_warp(g, index->view.dp, index->view.dc)) * g.warps_per_block > 220 * 1024)
        return set_error(HNSW_ERR_INVALID_ARGUMENT, "schedule needs more than 220 KB of shared memory per block");
    index->fixed = g;
    return HNSW_OK;
}

int hnsw_gpu_set_counters(hnsw_gpu_index* index, int enabled) {
    if (!index) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null index");
    index->counters = enabled != 0;
    return HNSW_OK;
}

int hnsw_gpu_read_counters(hnsw_gpu_index* index, uint32_t* host_out, size_t nq) {
    if (!index || !host_out) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> g(index->counters_mu);
    if (index->last_counters.size() < nq * 4) return set_error(HNSW_ERR_INVALID_ARGUMENT, "no counters for that many queries");
    std::memcpy(host_out, index->last_counters.data(), nq * 16);
    return HNSW_OK;
}


// Validates a host-buffer batch: the bound on max(ef, k) and the row stride.
static int check_batch(hnsw_gpu_index* gi, size_t nq, size_t dim, const hnsw_search_opts& o, uint32_t* ef_bound,
                       uint32_t* stride) {
    if (dim != gi->view.dim) {
        return set_error(HNSW_ERR_DIMENSION_MISMATCH, "dimension mismatch: expected " + std::to_string(gi->view.dim) +
                                                          ", got " + std::to_string(dim));
    }
    if (nq > 0x7FFFFFFFu) return set_error(HNSW_ERR_INVALID_ARGUMENT, "batch too large");
    uint32_t kmax = o.k, efmax = o.ef;
    if (o.ks)
        for (size_t i = 0; i < nq; ++i) kmax = std::max(kmax, o.ks[i]);
    else
        kmax = o.k;
    if (o.efs)
        for (size_t i = 0; i < nq; ++i) efmax = std::max(efmax, o.efs[i]);
    *ef_bound = std::max(kmax, efmax);
    if (*ef_bound > 65536) return set_error(HNSW_ERR_INVALID_ARGUMENT, "ef and k above 65536 are not supported on the device");
    *stride = o.out_stride ? o.out_stride : std::max<uint32_t>(kmax, 1);
    if (*stride < kmax) return set_error(HNSW_ERR_INVALID_ARGUMENT, "out_stride below k");
    if (o.filter_bits && o.filter_nbits == 0) return set_error(HNSW_ERR_INVALID_ARGUMENT, "filter bitmap has no bits");
    if (o.mode != HNSW_MODE_PLAIN && o.mode != HNSW_MODE_PERSISTENT && o.mode != HNSW_MODE_AUTO)
        return set_error(HNSW_ERR_INVALID_ARGUMENT, "unknown search mode");
    return HNSW_OK;
}

// Device copies of a host batch's inputs, staged on the slot's stream.
struct StagedBatch {
    const uint32_t* ks = nullptr;
    const uint32_t* efs = nullptr;
    const uint64_t* fbits = nullptr;
    const uint8_t* fused = nullptr;
    const uint32_t* fids = nullptr;
};

static int stage_batch(Slot* s, const float* queries, size_t nq, size_t dim, const hnsw_search_opts& o,
                       uint32_t stride, StagedBatch* out) {
    cudaStream_t st = s->stream;
    CU(s->q.ensure(nq * dim * 4), "cudaMalloc queries");
    CU(cudaMemcpyAsync(s->q.p, queries, nq * dim * 4, cudaMemcpyHostToDevice, st), "copy queries");
    const uint32_t* d_ks = nullptr;
    const uint32_t* d_efs = nullptr;
    const uint64_t* d_fb = nullptr;
    const uint8_t* d_fu = nullptr;
    if (o.ks) {
        CU(s->ks.ensure(nq * 4), "cudaMalloc ks");
        CU(cudaMemcpyAsync(s->ks.p, o.ks, nq * 4, cudaMemcpyHostToDevice, st), "copy ks");
        d_ks = s->ks.as<uint32_t>();
    }
    if (o.efs) {
        CU(s->efs.ensure(nq * 4), "cudaMalloc efs");
        CU(cudaMemcpyAsync(s->efs.p, o.efs, nq * 4, cudaMemcpyHostToDevice, st), "copy efs");
        d_efs = s->efs.as<uint32_t>();
    }
    const uint32_t* d_fi = nullptr;
    if (o.filter_bits) {
        const uint64_t words = (o.filter_nbits + 63) / 64;
        uint64_t bitmaps = nq;
        if (o.filter_ids) {
            uint32_t mx = 0;
            for (size_t i = 0; i < nq; ++i) mx = std::max(mx, o.filter_ids[i]);
            bitmaps = uint64_t(mx) + 1;
            CU(s->fids.ensure(nq * 4), "cudaMalloc filter ids");
            CU(cudaMemcpyAsync(s->fids.p, o.filter_ids, nq * 4, cudaMemcpyHostToDevice, st), "copy filter ids");
            d_fi = s->fids.as<uint32_t>();
        }
        const uint64_t total = o.filter_stride ? o.filter_stride * (bitmaps - 1) + words : words;
        CU(s->fbits.ensure(total * 8), "cudaMalloc filter");
        CU(cudaMemcpyAsync(s->fbits.p, o.filter_bits, total * 8, cudaMemcpyHostToDevice, st), "copy filter");
        d_fb = s->fbits.as<uint64_t>();
        if (o.filter_used) {
            CU(s->fused.ensure(nq), "cudaMalloc filter flags");
            CU(cudaMemcpyAsync(s->fused.p, o.filter_used, nq, cudaMemcpyHostToDevice, st), "copy filter flags");
            d_fu = s->fused.as<uint8_t>();
        }
    }
    CU(s->okeys.ensure(nq * stride * 8), "cudaMalloc out keys");
    CU(s->odist.ensure(nq * stride * 4), "cudaMalloc out dist");
    CU(s->ocount.ensure(nq * 4), "cudaMalloc out count");
    CU(s->ostatus.ensure(nq * 4), "cudaMalloc out status");
    out->ks = d_ks;
    out->efs = d_efs;
    out->fbits = d_fb;
    out->fused = d_fu;
    out->fids = d_fi;
    return HNSW_OK;
}

// The first non-OK query status of a finished batch becomes the call's error.
static int batch_status(const int32_t* out_status, size_t nq) {
    for (size_t i = 0; i < nq; ++i)
        if (out_status[i] != HNSW_OK) {
            const int32_t code = out_status[i];
            std::string msg = code == HNSW_ERR_NON_FINITE_VECTOR ? "vector contains NaN or infinite values"
                              : code == HNSW_ERR_ZERO_VECTOR     ? "zero vector has no direction under cosine distance"
                              : code == HNSW_ERR_QUANTIZATION_DISABLED
                                  ? "quantized search requested but quantization is not enabled"
                              : code == HNSW_ERR_SCRATCH_OVERFLOW ? "a query outgrew the device scratch"
                                                                  : "query failed";
            return set_error(code, msg);
        }
    return HNSW_OK;
}

int hnsw_gpu_search_batch(hnsw_gpu_index* gi, const float* queries, size_t nq, size_t dim,
                          const hnsw_search_opts* opts, uint64_t* out_keys, float* out_dist, uint32_t* out_count,
                          int32_t* out_status) {
    if (!gi || !opts) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    const hnsw_search_opts& o = *opts;
    uint32_t ef_bound = 0, stride = 0;
    int r = check_batch(gi, nq, dim, o, &ef_bound, &stride);
    if (r != HNSW_OK) return r;
    if (nq == 0) return HNSW_OK;
    if (!queries || !out_keys || !out_dist || !out_count || !out_status)
        return set_error(HNSW_ERR_INVALID_ARGUMENT, "null buffer");
    DeviceGuard dg(gi->device);
    TraceRange trace("hnsw.search_batch");
    Slot* s = nullptr;
    r = gi->slots.acquire(&s);
    if (r != HNSW_OK) return r;
    std::unique_ptr<Slot, std::function<void(Slot*)>> hold(s, [gi](Slot* p) { gi->slots.release(p); });
    cudaStream_t st = s->stream;
    StagedBatch sb;
    r = stage_batch(s, queries, nq, dim, o, stride, &sb);
    if (r != HNSW_OK) return r;
    r = enqueue_search(gi, s, s->q.as<float>(), nq, o, sb.ks, sb.efs, sb.fbits, sb.fused, sb.fids,
                       s->okeys.as<uint64_t>(), s->odist.as<float>(), s->ocount.as<uint32_t>(),
                       s->ostatus.as<int32_t>(), ef_bound, stride, st);
    if (r != HNSW_OK) return r;
    CU(cudaMemcpyAsync(out_count, s->ocount.p, nq * 4, cudaMemcpyDeviceToHost, st), "copy counts");
    CU(cudaMemcpyAsync(out_status, s->ostatus.p, nq * 4, cudaMemcpyDeviceToHost, st), "copy statuses");
    CU(cudaMemcpyAsync(out_keys, s->okeys.p, nq * stride * 8, cudaMemcpyDeviceToHost, st), "copy keys");
    CU(cudaMemcpyAsync(out_dist, s->odist.p, nq * stride * 4, cudaMemcpyDeviceToHost, st), "copy distances");
    CU(cudaStreamSynchronize(st), "search");
    if (gi->counters) {
        std::lock_guard<std::mutex> g(gi->counters_mu);
        gi->last_counters.resize(nq * 4);
        CU(cudaMemcpy(gi->last_counters.data(), s->counters.p, nq * 16, cudaMemcpyDeviceToHost), "copy counters");
    }
    return batch_status(out_status, nq);
}

int hnsw_gpu_clear_tuning(hnsw_gpu_index* gi) {
    if (!gi) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null index");
    std::lock_guard<std::mutex> l(gi->tune_mu);
    for (auto& t : gi->tuned) t = hnsw_gpu_index::Tuned();
    return HNSW_OK;
}

int hnsw_gpu_autotune(hnsw_gpu_index* gi, const float* queries, size_t nq, size_t dim, const hnsw_search_opts* opts,
                      uint32_t reps, hnsw_tune_entry* entries, size_t cap, size_t* written, hnsw_tune_entry* best) {
    if (written) *written = 0;
    if (!gi || !opts) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    const hnsw_search_opts& o = *opts;
    uint32_t ef_bound = 0, stride = 0;
    int r = check_batch(gi, nq, dim, o, &ef_bound, &stride);
    if (r != HNSW_OK) return r;
    if (nq == 0 || !queries) return set_error(HNSW_ERR_INVALID_ARGUMENT, "the autotuner needs a sample batch");
    if (reps == 0) reps = 3;
    if (reps > 50) return set_error(HNSW_ERR_INVALID_ARGUMENT, "at most 50 timed runs per schedule");
    DeviceGuard dg(gi->device);
    TraceRange trace("hnsw.autotune");
    Slot* s = nullptr;
    r = gi->slots.acquire(&s);
    if (r != HNSW_OK) return r;
    std::unique_ptr<Slot, std::function<void(Slot*)>> hold(s, [gi](Slot* p) { gi->slots.release(p); });
    cudaStream_t st = s->stream;
    StagedBatch sb;
    r = stage_batch(s, queries, nq, dim, o, stride, &sb);
    if (r != HNSW_OK) return r;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    CU(cudaEventCreate(&ev[0]), "cudaEventCreate");
    if (cudaEventCreate(&ev[1]) != cudaSuccess) {
        cudaEventDestroy(ev[0]);
        return cuda_fail(cudaGetLastError(), "cudaEventCreate");
    }
    std::unique_ptr<cudaEvent_t, void (*)(cudaEvent_t*)> evs(ev, [](cudaEvent_t* e) {
        cudaEventDestroy(e[0]);
        cudaEventDestroy(e[1]);
    });
    // Coordinate descent per mode from the heuristic's choice: the
    // cold-list variant (persistent), warps per block {1,2,4,8}, visited hash
    // {16,24,32,40,48,64} entries per result slot (multiples of 64 within
    // 1024..32768),
    // staged rows {0,16,32}, then warps per block again; a change is kept
    // when it is faster. ef_cap is the bucket's bound.
    const uint32_t ef_cap = std::min<uint32_t>(1024, std::max<uint32_t>(32, round_up(ef_bound, 32)));
    const uint32_t row_bytes = (o.quantized && gi->view.quantized) ? gi->view.dc : gi->view.dp * 4;
    const bool filtered = o.filter_bits != nullptr;
    struct Trial {
        SearchGeometry g;
        int32_t mode;
        int32_t heuristic;
        float ms;
    };
    std::vector<Trial> trials;
    std::vector<float> times(reps);
    auto same = [](const SearchGeometry& x, const SearchGeometry& y) {
        return x.ef_cap == y.ef_cap && x.cand_cap == y.cand_cap && x.hash_cap == y.hash_cap &&
               x.warps_per_block == y.warps_per_block && x.stage_rows == y.stage_rows && x.cold == y.cold;
    };
    // Times one schedule; returns false on an error (status in r).
    auto timed = [&](const SearchGeometry& g, int32_t mode, int32_t heuristic, float* ms) {
        hnsw_search_opts ot = o;
        ot.mode = mode;
        auto run = [&]() {
            return enqueue_search(gi, s, s->q.as<float>(), nq, ot, sb.ks, sb.efs, sb.fbits, sb.fused, sb.fids,
                                  s->okeys.as<uint64_t>(), s->odist.as<float>(), s->ocount.as<uint32_t>(),
                                  s->ostatus.as<int32_t>(), ef_bound, stride, st, &g);
        };
        r = run();  // warm-up; sizes every buffer
        if (r != HNSW_OK) return false;
        for (uint32_t i = 0; i < reps; ++i) {
            cudaError_t e = cudaEventRecord(ev[0], st);
            if (e == cudaSuccess) {
                r = run();
                if (r != HNSW_OK) return false;
                e = cudaEventRecord(ev[1], st);
            }
            if (e == cudaSuccess) e = cudaEventSynchronize(ev[1]);
            if (e == cudaSuccess) e = cudaEventElapsedTime(&times[i], ev[0], ev[1]);
            if (e != cudaSuccess) {
                r = cuda_fail(e, "autotune run");
                return false;
            }
        }
        std::vector<float> sorted = times;
        std::sort(sorted.begin(), sorted.end());
        *ms = sorted[reps / 2];
        trials.push_back({g, mode, heuristic, *ms});
        return true;
    };
    for (int32_t mode : {HNSW_MODE_PLAIN, HNSW_MODE_PERSISTENT}) {
        const bool pers = mode == HNSW_MODE_PERSISTENT;
        SearchGeometry cur = pick_geometry(ef_bound, gi->view.dp, gi->view.dc, pers, filtered, gi->view.n);
        cur.stage_row_bytes = cur.stage_rows ? row_bytes : 0;
        float best_ms = 0.0f;
        if (!timed(cur, mode, 1, &best_ms)) return r;
        auto consider = [&](SearchGeometry g) {
            g.stage_row_bytes = g.stage_rows ? row_bytes : 0;
            set_hash_tags(g, gi->view.n, g_visit_tag_bits.load());
            if (size_t(geometry_bytes_per_warp(g, gi->view.dp, gi->view.dc)) * g.warps_per_block > 220 * 1024)
                return true;
            for (const Trial& t : trials)
                if (t.mode == mode && same(t.g, g)) return true;
            float ms = 0.0f;
            if (!timed(g, mode, 0, &ms)) return false;
            if (ms < best_ms) {
                best_ms = ms;
                cur = g;
            }
            return true;
        };
        if (pers) {
            SearchGeometry g = cur;
            g.cold ^= 1u;
            if (!consider(g)) return r;
        }
        for (int pass = 0; pass < 2; ++pass) {
            for (uint32_t wpb : {1u, 2u, 4u, 8u}) {
                SearchGeometry g = cur;
                g.warps_per_block = wpb;
                if (!consider(g)) return r;
            }
            if (pass == 1) break;
            // Hash sizes need not be powers of two: 24 or 40 entries per
            // result slot can fit one more warp per SM than 32 or 48 (a
            // power of two may store 16-bit tags, which halves its bytes).
            for (uint32_t per : {16u, 24u, 32u, 40u, 48u, 64u, 128u}) {
                const uint32_t hc = std::min<uint32_t>(32768, std::max<uint32_t>(1024, round_up(ef_cap * per, 64)));
                SearchGeometry g = cur;
                g.ef_cap = ef_cap;
                g.hash_cap = hc;
                if (!consider(g)) return r;
            }
            for (uint32_t stage : {0u, 16u, 32u}) {
                SearchGeometry g = cur;
                g.stage_rows = stage;
                if (!consider(g)) return r;
            }
        }
    }
    const Trial* win[2] = {nullptr, nullptr};
    for (const Trial& t : trials)
        if (!win[t.mode] || t.ms < win[t.mode]->ms) win[t.mode] = &t;
    const Trial* top = win[0]->ms <= win[1]->ms ? win[0] : win[1];
    {
        std::lock_guard<std::mutex> l(gi->tune_mu);
        hnsw_gpu_index::Tuned& slot = gi->tuned[tune_bucket(ef_bound)];
        slot.geo[0] = win[0]->g;
        slot.geo[1] = win[1]->g;
        slot.mode = top->mode;
    }
    auto fill = [](const Trial& t, hnsw_tune_entry* e) {
        e->schedule.ef_cap = t.g.ef_cap;
        e->schedule.cand_cap = t.g.cand_cap;
        e->schedule.hash_cap = t.g.hash_cap;
        e->schedule.warps_per_block = t.g.warps_per_block;
        e->schedule.cold_chunks = t.g.cold_chunks;
        e->schedule.stage_rows = t.g.stage_rows;
        e->schedule.cold = t.g.cold;
        e->mode = t.mode;
        e->heuristic = t.heuristic;
        e->ms = t.ms;
    };
    if (entries) {
        const size_t n = std::min(cap, trials.size());
        for (size_t i = 0; i < n; ++i) fill(trials[i], &entries[i]);
        if (written) *written = n;
    }
    if (best) fill(*top, best);
    return HNSW_OK;
}

int hnsw_gpu_search_batch_device(hnsw_gpu_index* gi, const float* d_queries, size_t nq, size_t dim,
                                 const hnsw_search_opts* o, uint64_t* d_keys, float* d_dist, uint32_t* d_count,
                                 int32_t* d_status, void* stream) {
    if (!gi || !o) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    if (dim != gi->view.dim) return set_error(HNSW_ERR_DIMENSION_MISMATCH, "dimension mismatch");
    if (nq == 0) return HNSW_OK;
    const uint32_t ef_bound = std::max(o->k, o->ef);
    const uint32_t stride = o->out_stride ? o->out_stride : std::max<uint32_t>(o->k, 1);
    DeviceGuard dg(gi->device);
    TraceRange trace("hnsw.search_batch_device");
    std::lock_guard<std::mutex> lock(gi->dev_mu);
    if (!gi->dev_slot) {
        Slot* s = nullptr;
        int r = gi->slots.acquire(&s);
        if (r != HNSW_OK) return r;
        gi->dev_slot.reset(s);
        CU(cudaEventCreateWithFlags(&gi->dev_done, cudaEventDisableTiming), "cudaEventCreate");
        CU(cudaEventRecord(gi->dev_done, s->stream), "cudaEventRecord");
    }
    Slot* s = gi->dev_slot.get();
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->stream;
    // The slot's buffers may still be in use by the previous call on another stream.
    CU(cudaStreamWaitEvent(st, gi->dev_done, 0), "cudaStreamWaitEvent");
    int r = enqueue_search(gi, s, d_queries, nq, *o, o->ks, o->efs, o->filter_bits, o->filter_used, o->filter_ids,
                           d_keys, d_dist, d_count, d_status, ef_bound, stride, st);
    CU(cudaEventRecord(gi->dev_done, st), "cudaEventRecord");
    return r;
}

struct hnsw_gpu_graph {
    hnsw_gpu_index* index = nullptr;
    Slot* slot = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

// Captures memset + search + retry for a fixed batch (relaxed capture mode;
// a warm-up enqueue first sizes every buffer, so the captured call allocates
// nothing).
int hnsw_gpu_graph_create(hnsw_gpu_index* gi, const float* d_queries, size_t nq, size_t dim,
                          const hnsw_search_opts* o, uint64_t* d_keys, float* d_dist, uint32_t* d_count,
                          int32_t* d_status, hnsw_gpu_graph** out) {
    if (!gi || !o || !out) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (dim != gi->view.dim) return set_error(HNSW_ERR_DIMENSION_MISMATCH, "dimension mismatch");
    if (nq == 0) return set_error(HNSW_ERR_INVALID_ARGUMENT, "empty batch");
    DeviceGuard dg(gi->device);
    std::unique_ptr<hnsw_gpu_graph> g(new hnsw_gpu_graph());
    g->index = gi;
    int r = gi->slots.acquire(&g->slot);
    if (r != HNSW_OK) return r;
    cudaStream_t st = g->slot->stream;
    const uint32_t ef_bound = std::max(o->k, o->ef);
    const uint32_t stride = o->out_stride ? o->out_stride : std::max<uint32_t>(o->k, 1);
    auto enqueue = [&]() {
        return enqueue_search(gi, g->slot, d_queries, nq, *o, o->ks, o->efs, o->filter_bits, o->filter_used,
                              o->filter_ids, d_keys, d_dist, d_count, d_status, ef_bound, stride, st);
    };
    r = enqueue();
    if (r != HNSW_OK) {
        gi->slots.release(g->slot);
        return r;
    }
    cudaError_t e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) {
        gi->slots.release(g->slot);
        return cuda_fail(e, "graph capture");
    }
    r = enqueue();
    e = cudaStreamEndCapture(st, &g->graph);
    if (r != HNSW_OK || e != cudaSuccess) {
        if (g->graph) cudaGraphDestroy(g->graph);
        gi->slots.release(g->slot);
        return r != HNSW_OK ? r : cuda_fail(e, "graph capture");
    }
    e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g->graph);
        gi->slots.release(g->slot);
        return cuda_fail(e, "graph instantiate");
    }
    *out = g.release();
    return HNSW_OK;
}

int hnsw_gpu_graph_launch(hnsw_gpu_graph* g, void* stream) {
    if (!g) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null graph");
    DeviceGuard dg(g->index->device);
    TraceRange trace("hnsw.graph_launch");
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : g->slot->stream;
    CU(cudaGraphLaunch(g->exec, st), "graph launch");
    return HNSW_OK;
}

void hnsw_gpu_graph_destroy(hnsw_gpu_graph* g) {
    if (!g) return;
    DeviceGuard dg(g->index->device);
    cudaStreamSynchronize(g->slot->stream);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    g->index->slots.release(g->slot);
    delete g;
}

// ------------------------------------------------------------------------
// Brute force
// ------------------------------------------------------------------------
int hnsw_gpu_brute_open(const float* vectors, const uint64_t* keys, size_t n, size_t dim, int metric, int device,
                        hnsw_gpu_brute** out) {
    if (!out) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null output handle");
    *out = nullptr;
    if (dim == 0 || dim > kMaxDim) return set_error(HNSW_ERR_INVALID_DIMENSION, "invalid dimension");
    if (metric < 0 || metric > 2) return set_error(HNSW_ERR_INVALID_ARGUMENT, "unknown metric");
    if (n && !vectors) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null vectors");
    if (n > 0xFFFFFFF0ull) return set_error(HNSW_ERR_CAPACITY_EXCEEDED, "too many vectors");
    // insert_batch: prepare every row, keys unique (src/brute.rs:103-115).
    const uint32_t dp = round_up(uint32_t(dim), 32);
    std::vector<float> rows(std::max<size_t>(n, 1) * dp, 0.0f);
    for (size_t i = 0; i < n; ++i) {
        double norm;
        int s = check_vector(vectors + i * dim, dim, &norm);
        if (s) return set_error(s, "vector contains NaN or infinite values");
        if (metric == HNSW_METRIC_COSINE) {
            if (norm == 0.0) return set_error(HNSW_ERR_ZERO_VECTOR, "zero vector has no direction under cosine distance");
            double inv = 1.0 / std::sqrt(norm);
            for (size_t j = 0; j < dim; ++j) rows[i * dp + j] = float(double(vectors[i * dim + j]) * inv);
        } else {
            std::memcpy(&rows[i * dp], vectors + i * dim, dim * 4);
        }
    }
    std::vector<uint64_t> kv(std::max<size_t>(n, 1));
    for (size_t i = 0; i < n; ++i) kv[i] = keys ? keys[i] : uint64_t(i);
    if (keys) {
        std::vector<uint64_t> sorted(kv.begin(), kv.begin() + n);
        std::sort(sorted.begin(), sorted.end());
        auto it = std::adjacent_find(sorted.begin(), sorted.end());
        if (it != sorted.end()) return set_error(HNSW_ERR_DUPLICATE_KEY, "key " + std::to_string(*it) + " is already present");
    }
    DeviceGuard dg(device);
    std::unique_ptr<hnsw_gpu_brute> b(new hnsw_gpu_brute());
    b->device = device;
    cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device);
    {
        double mx = 0.0;
        for (size_t i = 0; i < n; ++i) {
            double s2 = 0.0;
            for (size_t j = 0; j < dim; ++j) s2 += double(rows[i * dp + j]) * double(rows[i * dp + j]);
            mx = std::max(mx, s2);
        }
        b->max_xnorm = float(std::sqrt(mx) * (1.0 + 1e-6));
    }
    b->n = uint32_t(n);
    b->dim = uint32_t(dim);
    b->dp = dp;
    b->metric = metric;
    CU(b->base.ensure(rows.size() * 4), "cudaMalloc base");
    CU(cudaMemcpy(b->base.p, rows.data(), rows.size() * 4, cudaMemcpyHostToDevice), "copy base");
    CU(b->keys.ensure(kv.size() * 8), "cudaMalloc keys");
    CU(cudaMemcpy(b->keys.p, kv.data(), kv.size() * 8, cudaMemcpyHostToDevice), "copy keys");
    CU(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream");
    *out = b.release();
    return HNSW_OK;
}

void hnsw_gpu_brute_close(hnsw_gpu_brute* brute) { delete brute; }

// Tensor-core brute force: BF16 (1 term) or compensated BF16 (3 terms)
// scoring with FP32 accumulation, then exact FP32 re-ranking.
//   1. queries: validate/normalise (FP32), split into BF16 operand rows;
//   2. sample pass: dense approximate distances to the first rows; the k-th
//      smallest plus 2E (E bounds |approximate - FP32| distance) is a
//      threshold every true top-k row passes;
//   3. candidate pass over all rows: (row, approximate distance) <= threshold;
//   4. a tighter threshold: k-th smallest candidate + 2E;
//   5. exact FP32 distances (reference order) of those candidates, top-k by
//      (distance, key). Queries whose candidate list overflowed are re-run
//      with the exact FP32 kernels.
static int brute_search_tensor(hnsw_gpu_brute* b, const float* queries, size_t nq, uint32_t k, int precision,
                               uint64_t* out_keys, float* out_dist, uint32_t* out_count, int32_t* out_status) {
    std::lock_guard<std::mutex> lock(b->mu);
    DeviceGuard dg(b->device);
    TraceRange trace("hnsw.brute_search_tensor");
    cudaStream_t st = b->stream;
    const int terms = precision == HNSW_PRECISION_BF16X3 ? 3 : 1;
    const int ti = terms == 3 ? 1 : 0;
    const uint32_t kp = tc_k_padded(b->dim, terms);
    const uint32_t np = tc_rows_padded(b->n, false);
    const bool pairs = b->tc_pairs != 0;
    const uint32_t qp = tc_rows_padded(uint32_t(nq), true, pairs);
    if (b->bop_kp[ti] != kp) {
        CU(b->bop[ti].ensure(size_t(np) * kp * 2), "cudaMalloc BF16 rows");
        CU(tc_split(b->base.as<float>(), b->n, b->dim, b->dp, b->bop[ti].as<__nv_bfloat16>(), np, kp, terms, false, st),
           "split rows");
        b->bop_kp[ti] = kp;
    }
    if (b->metric == HNSW_METRIC_L2 && b->xnorm2.bytes < size_t(np) * 4) {
        CU(b->xnorm2.ensure(size_t(np) * 4), "cudaMalloc row norms");
        CU(tc_row_norms(b->base.as<float>(), b->n, b->dim, b->dp, b->xnorm2.as<float>(), st), "row norms");
    }
    BruteArgs a;
    a.base = b->base.as<float>();
    a.keys = b->keys.as<uint64_t>();
    a.n = b->n;
    a.dim = b->dim;
    a.dp = b->dp;
    a.metric = b->metric;
    a.nq = uint32_t(nq);
    a.k = k;
    if (!b->ev[0])
        for (cudaEvent_t& e : b->ev) CU(cudaEventCreate(&e), "cudaEventCreate");
    CU(b->q.ensure(nq * b->dim * 4), "cudaMalloc queries");
    CU(cudaMemcpyAsync(b->q.p, queries, nq * b->dim * 4, cudaMemcpyHostToDevice, st), "copy queries");
    CU(b->qprep.ensure(size_t(qp) * b->dp * 4), "cudaMalloc qprep");
    CU(b->okeys.ensure(nq * size_t(k) * 8), "cudaMalloc out keys");
    CU(b->odist.ensure(nq * size_t(k) * 4), "cudaMalloc out dist");
    CU(b->ocount.ensure(nq * 4), "cudaMalloc out count");
    CU(b->ostatus.ensure(nq * 4), "cudaMalloc out status");
    a.queries = b->q.as<float>();
    a.qprep = b->qprep.as<float>();
    a.out_keys = b->okeys.as<uint64_t>();
    a.out_dist = b->odist.as<float>();
    a.out_count = b->ocount.as<uint32_t>();
    a.out_status = b->ostatus.as<int32_t>();
    CU(cudaEventRecord(b->ev[0], st), "event");
    CU(launch_brute_prep(a, st), "query prep");
    // Query norms (L2 epilogue and margins) and BF16 query operands.
    CU(b->qnorm2.ensure(size_t(qp) * 4), "cudaMalloc query norms");
    CU(tc_row_norms(a.qprep, uint32_t(nq), b->dim, b->dp, b->qnorm2.as<float>(), st), "query norms");
    CU(b->aop.ensure(size_t(qp) * kp * 2), "cudaMalloc BF16 queries");
    CU(tc_split(a.qprep, uint32_t(nq), b->dim, b->dp, b->aop.as<__nv_bfloat16>(), qp, kp, terms, true, st), "split queries");
    const double u24 = 5.9604644775390625e-8;
    const double eps = terms == 3 ? (3.1 * 1.52587890625e-5 + double(kp + b->dim + 8) * u24)
                                  : (2.0 * 3.90625e-3 + 1.52587890625e-5 + double(kp + b->dim + 8) * u24);
    CU(b->margin.ensure(size_t(qp) * 4), "cudaMalloc margins");
    CU(tc_margins(b->qnorm2.as<float>(), uint32_t(nq), b->max_xnorm, float(eps), b->metric, b->dim,
                  b->margin.as<float>(), st),
       "margins");
    CU(b->err.ensure(16), "cudaMalloc error word");
    CU(cudaMemsetAsync(b->err.p, 0, 16, st), "memset error word");
    // Sample pass.
    CU(cudaEventRecord(b->ev[1], st), "event");
    const uint32_t sample_rows = std::min<uint32_t>(np, 16384);
    CU(b->dense.ensure(size_t(qp) * sample_rows * 4), "cudaMalloc sample");
    CU(b->thr1.ensure(size_t(qp) * 4), "cudaMalloc thresholds");
    CU(b->thr2.ensure(size_t(qp) * 4), "cudaMalloc thresholds");
    TcScoreArgs t;
    t.terms = terms;
    t.nq = uint32_t(nq);
    t.n = b->n;
    t.metric = b->metric;
    t.qnorm2 = b->qnorm2.as<float>();
    t.xnorm2 = b->metric == HNSW_METRIC_L2 ? b->xnorm2.as<float>() : nullptr;
    t.err = b->err.as<uint32_t>();
    t.wait_budget = b->wait_budget;
    t.stall = b->stall;
    t.pairs = pairs ? 1u : 0u;
    t.n_tile_begin = 0;
    t.n_tile_end = sample_rows / 256;
    t.dense = b->dense.as<float>();
    t.row0 = 0;
    t.ld = sample_rows;
    CU(tc_score(b->aop.as<__nv_bfloat16>(), qp, b->bop[ti].as<__nv_bfloat16>(), np, kp, t, b->num_sms, st), "sample pass");
    const uint32_t kk = std::min<uint32_t>(k, b->n);
    CU(tc_kth_threshold(b->dense.as<float>(), sample_rows, nullptr, nullptr, 0, uint32_t(nq), kk, b->margin.as<float>(),
                        b->thr1.as<float>(), st),
       "sample threshold");
    // Candidate pass.
    const uint32_t cap = 32768;
    CU(b->ccount.ensure(size_t(qp) * 4), "cudaMalloc candidate counts");
    CU(b->cand.ensure(size_t(nq) * cap * 8), "cudaMalloc candidates");
    CU(cudaMemsetAsync(b->ccount.p, 0, size_t(qp) * 4, st), "memset candidate counts");
    t.dense = nullptr;
    t.n_tile_begin = 0;
    t.n_tile_end = np / 256;
    t.thr = b->thr1.as<float>();
    t.cand_count = b->ccount.as<uint32_t>();
    t.cand = b->cand.as<uint64_t>();
    t.cand_cap = cap;
    CU(cudaEventRecord(b->ev[2], st), "event");
    CU(tc_score(b->aop.as<__nv_bfloat16>(), qp, b->bop[ti].as<__nv_bfloat16>(), np, kp, t, b->num_sms, st),
       "candidate pass");
    CU(cudaEventRecord(b->ev[3], st), "event");
    CU(tc_kth_threshold(nullptr, 0, b->ccount.as<uint32_t>(), b->cand.as<uint64_t>(), cap, uint32_t(nq), kk,
                        b->margin.as<float>(), b->thr2.as<float>(), st),
       "candidate threshold");
    CU(launch_brute_rerank(a, b->cand.as<uint64_t>(), b->ccount.as<uint32_t>(), cap, b->thr2.as<float>(), st),
       "re-rank");
    CU(cudaEventRecord(b->ev[4], st), "event");
    uint32_t err = 0;
    CU(cudaMemcpyAsync(&err, b->err.p, 4, cudaMemcpyDeviceToHost, st), "copy error word");
    CU(cudaMemcpyAsync(out_count, a.out_count, nq * 4, cudaMemcpyDeviceToHost, st), "copy counts");
    CU(cudaMemcpyAsync(out_status, a.out_status, nq * 4, cudaMemcpyDeviceToHost, st), "copy statuses");
    CU(cudaMemcpyAsync(out_keys, a.out_keys, nq * size_t(k) * 8, cudaMemcpyDeviceToHost, st), "copy keys");
    CU(cudaMemcpyAsync(out_dist, a.out_dist, nq * size_t(k) * 4, cudaMemcpyDeviceToHost, st), "copy distances");
    CU(cudaStreamSynchronize(st), "tensor brute force");
    for (int i = 0; i < 4; ++i) cudaEventElapsedTime(&b->last_ms[i], b->ev[i], b->ev[i + 1]);
    if (err) return set_error(HNSW_ERR_TIMEOUT, "tensor-core scoring: a bounded wait ran out");
    // Queries whose candidate list overflowed: exact FP32 kernels.
    std::vector<uint32_t> redo;
    for (size_t i = 0; i < nq; ++i)
        if (out_status[i] == HNSW_ERR_SCRATCH_OVERFLOW) redo.push_back(uint32_t(i));
    if (!redo.empty()) {
        std::vector<float> sub(redo.size() * b->dim);
        for (size_t j = 0; j < redo.size(); ++j)
            std::memcpy(&sub[j * b->dim], queries + size_t(redo[j]) * b->dim, b->dim * 4);
        std::vector<uint64_t> sk(redo.size() * k);
        std::vector<float> sd(redo.size() * k);
        std::vector<uint32_t> sc(redo.size());
        std::vector<int32_t> ss(redo.size());
        b->mu.unlock();
        int r = hnsw_gpu_brute_search_batch(b, sub.data(), redo.size(), b->dim, k, HNSW_PRECISION_FP32, sk.data(),
                                            sd.data(), sc.data(), ss.data());
        b->mu.lock();
        if (r != HNSW_OK) return r;
        for (size_t j = 0; j < redo.size(); ++j) {
            const size_t i = redo[j];
            out_count[i] = sc[j];
            out_status[i] = ss[j];
            std::memcpy(out_keys + i * k, &sk[j * k], size_t(k) * 8);
            std::memcpy(out_dist + i * k, &sd[j * k], size_t(k) * 4);
        }
    }
    {
        std::vector<uint32_t> counts(nq);
        if (cudaMemcpy(counts.data(), b->ccount.p, nq * 4, cudaMemcpyDeviceToHost) == cudaSuccess) {
            uint64_t total = 0;
            for (uint32_t c : counts) total += c;
            b->last_candidates = total;
            b->last_queries = nq;
        }
    }
    for (size_t i = 0; i < nq; ++i)
        if (out_status[i] != HNSW_OK) return set_error(out_status[i], "query failed validation");
    return HNSW_OK;
}

// Exact FP32 brute force (reference kernel order), optionally filtered.
static int brute_search_fp32(hnsw_gpu_brute* b, const float* queries, size_t nq, size_t dim, uint32_t k,
                             const hnsw_brute_filter* f, uint64_t* out_keys, float* out_dist, uint32_t* out_count,
                             int32_t* out_status) {
    std::lock_guard<std::mutex> lock(b->mu);
    DeviceGuard dg(b->device);
    TraceRange trace("hnsw.brute_search_fp32");
    cudaStream_t st = b->stream;
    const uint32_t kk = std::max<uint32_t>(k, 1);
    BruteArgs a;
    a.base = b->base.as<float>();
    a.keys = b->keys.as<uint64_t>();
    a.n = b->n;
    a.dim = b->dim;
    a.dp = b->dp;
    a.metric = b->metric;
    a.nq = uint32_t(nq);
    a.k = k;
    a.tiles = std::max<uint32_t>(1, std::min<uint32_t>(64, (b->n + 8191) / 8192));
    CU(b->q.ensure(nq * dim * 4), "cudaMalloc queries");
    CU(cudaMemcpyAsync(b->q.p, queries, nq * dim * 4, cudaMemcpyHostToDevice, st), "copy queries");
    CU(b->qprep.ensure(nq * b->dp * 4), "cudaMalloc qprep");
    CU(b->part.ensure(size_t(nq) * a.tiles * kk * 8), "cudaMalloc partial");
    CU(b->okeys.ensure(nq * kk * 8), "cudaMalloc out keys");
    CU(b->odist.ensure(nq * kk * 4), "cudaMalloc out dist");
    CU(b->ocount.ensure(nq * 4), "cudaMalloc out count");
    CU(b->ostatus.ensure(nq * 4), "cudaMalloc out status");
    a.queries = b->q.as<float>();
    a.qprep = b->qprep.as<float>();
    a.part = b->part.as<uint64_t>();
    a.out_keys = b->okeys.as<uint64_t>();
    a.out_dist = b->odist.as<float>();
    a.out_count = b->ocount.as<uint32_t>();
    a.out_status = b->ostatus.as<int32_t>();
    if (f && f->bits) {
        const uint64_t words = (f->nbits + 63) / 64;
        uint64_t bitmaps = f->stride ? nq : 1;
        if (f->ids) {
            uint32_t mx = 0;
            for (size_t i = 0; i < nq; ++i) mx = std::max(mx, f->ids[i]);
            bitmaps = uint64_t(mx) + 1;
            CU(b->fids.ensure(nq * 4), "cudaMalloc filter ids");
            CU(cudaMemcpyAsync(b->fids.p, f->ids, nq * 4, cudaMemcpyHostToDevice, st), "copy filter ids");
            a.filter_ids = b->fids.as<uint32_t>();
        }
        const uint64_t total = f->stride ? f->stride * (bitmaps - 1) + words : words;
        CU(b->fbits.ensure(total * 8), "cudaMalloc filter");
        CU(cudaMemcpyAsync(b->fbits.p, f->bits, total * 8, cudaMemcpyHostToDevice, st), "copy filter");
        a.filter_bits = b->fbits.as<uint64_t>();
        a.filter_nbits = f->nbits;
        a.filter_stride = f->stride;
        a.filter_by_row = f->by_row;
        if (f->used) {
            CU(b->fused.ensure(nq), "cudaMalloc filter flags");
            CU(cudaMemcpyAsync(b->fused.p, f->used, nq, cudaMemcpyHostToDevice, st), "copy filter flags");
            a.filter_used = b->fused.as<uint8_t>();
        }
    }
    CU(launch_brute_fp32(a, st), "brute kernel");
    CU(cudaMemcpyAsync(out_count, b->ocount.p, nq * 4, cudaMemcpyDeviceToHost, st), "copy counts");
    CU(cudaMemcpyAsync(out_status, b->ostatus.p, nq * 4, cudaMemcpyDeviceToHost, st), "copy statuses");
    if (k) {
        CU(cudaMemcpyAsync(out_keys, b->okeys.p, nq * size_t(k) * 8, cudaMemcpyDeviceToHost, st), "copy keys");
        CU(cudaMemcpyAsync(out_dist, b->odist.p, nq * size_t(k) * 4, cudaMemcpyDeviceToHost, st), "copy distances");
    }
    CU(cudaStreamSynchronize(st), "brute search");
    for (size_t i = 0; i < nq; ++i)
        if (out_status[i] != HNSW_OK) return set_error(out_status[i], "query failed validation");
    return HNSW_OK;
}

int hnsw_gpu_brute_search_batch(hnsw_gpu_brute* b, const float* queries, size_t nq, size_t dim, uint32_t k,
                                int precision, uint64_t* out_keys, float* out_dist, uint32_t* out_count,
                                int32_t* out_status) {
    if (!b) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null handle");
    if (dim != b->dim) return set_error(HNSW_ERR_DIMENSION_MISMATCH, "dimension mismatch");
    if (nq == 0) return HNSW_OK;
    if (precision < HNSW_PRECISION_FP32 || precision > HNSW_PRECISION_BF16X3)
        return set_error(HNSW_ERR_INVALID_ARGUMENT, "unknown precision");
    if (k > 1024) return set_error(HNSW_ERR_INVALID_ARGUMENT, "k above 1024 is not supported on the device");
    if (precision != HNSW_PRECISION_FP32 && b->n > 0 && k > 0)
        return brute_search_tensor(b, queries, nq, k, precision, out_keys, out_dist, out_count, out_status);
    return brute_search_fp32(b, queries, nq, dim, k, nullptr, out_keys, out_dist, out_count, out_status);
}

int hnsw_gpu_brute_search_filtered(hnsw_gpu_brute* b, const float* queries, size_t nq, size_t dim, uint32_t k,
                                   const hnsw_brute_filter* filter, uint64_t* out_keys, float* out_dist,
                                   uint32_t* out_count, int32_t* out_status) {
    if (!b) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null handle");
    if (dim != b->dim) return set_error(HNSW_ERR_DIMENSION_MISMATCH, "dimension mismatch");
    if (nq == 0) return HNSW_OK;
    if (k > 1024) return set_error(HNSW_ERR_INVALID_ARGUMENT, "k above 1024 is not supported on the device");
    if (filter && filter->bits && filter->nbits == 0)
        return set_error(HNSW_ERR_INVALID_ARGUMENT, "filter bitmap has no bits");
    if (!queries || (k && (!out_keys || !out_dist)) || !out_count || !out_status)
        return set_error(HNSW_ERR_INVALID_ARGUMENT, "null buffer");
    return brute_search_fp32(b, queries, nq, dim, k, filter, out_keys, out_dist, out_count, out_status);
}

int hnsw_gpu_brute_stats(const hnsw_gpu_brute* b, hnsw_brute_stats* out) {
    if (!b || !out) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    out->candidates = b->last_candidates;
    out->queries = b->last_queries;
    out->prep_ms = b->last_ms[0];
    out->sample_ms = b->last_ms[1];
    out->score_ms = b->last_ms[2];
    out->rerank_ms = b->last_ms[3];
    return HNSW_OK;
}

// For callers that must not allocate device memory once they are running:
// all scratch comes from a fixed 8 MiB array compiled into the library.
int hnsw_gpu_brute_set_wait_limits(hnsw_gpu_brute* b, uint64_t budget_cycles, int inject_stall) {
    if (!b) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null handle");
    std::lock_guard<std::mutex> lock(b->mu);
    b->wait_budget = budget_cycles == 0 ? 4000000000ll
                                        : (long long)std::min<uint64_t>(budget_cycles, uint64_t(1) << 62);
    b->stall = inject_stall ? 1u : 0u;
    return HNSW_OK;
}

int hnsw_gpu_brute_set_pairs(hnsw_gpu_brute* b, int enabled) {
    if (!b) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null handle");
    std::lock_guard<std::mutex> lock(b->mu);
    b->tc_pairs = enabled ? 1u : 0u;
    return HNSW_OK;
}

void hnsw_gpu_debug_fail_allocations(int count) { g_fail_allocations.store(count > 0 ? count : 0); }

void hnsw_gpu_debug_visit_tags(int mode) { g_visit_tag_bits.store(mode < 0 ? -1 : std::min(mode, 32)); }

int hnsw_gpu_check_word(hnsw_gpu_index* gi, uint32_t out[2], int clear) {
    if (!gi || !out) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    out[0] = out[1] = 0;
    if (!gi->chk.p) return HNSW_OK;
    DeviceGuard dg(gi->device);
    CU(cudaDeviceSynchronize(), "check word");
    CU(cudaMemcpy(out, gi->chk.p, 8, cudaMemcpyDeviceToHost), "copy check word");
    if (clear) CU(cudaMemset(gi->chk.p, 0, 16), "clear check word");
    return HNSW_OK;
}

int hnsw_gpu_checked_build(void) {
#ifdef HNSW_DEVICE_CHECKS
    return 1;
#else
    return 0;
#endif
}

int hnsw_gpu_brute_search_batch_noalloc(hnsw_gpu_brute* b, const float* d_queries, size_t nq, size_t dim,
                                        uint32_t k, uint64_t* d_keys, float* d_dist, uint32_t* d_count,
                                        int32_t* d_status, void* stream) {
    if (!b) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null handle");
    if (dim != b->dim) return set_error(HNSW_ERR_DIMENSION_MISMATCH, "dimension mismatch");
    if (nq == 0) return HNSW_OK;
    if (!d_queries || !d_count || !d_status || (k && (!d_keys || !d_dist)))
        return set_error(HNSW_ERR_INVALID_ARGUMENT, "null buffer");
    if (k > 1024) return set_error(HNSW_ERR_INVALID_ARGUMENT, "k above 1024 is not supported on the device");
    if (nq > 0x7FFFFFFFu) return set_error(HNSW_ERR_INVALID_ARGUMENT, "batch too large");
    DeviceGuard dg(b->device);
    void* scratch = nullptr;
    CU(noalloc_scratch_address(&scratch), "no-alloc scratch address");
    const uint32_t kk = std::max<uint32_t>(1, std::min<uint32_t>(k, b->n ? b->n : 1));
    const uint32_t want = std::max<uint32_t>(1, std::min<uint32_t>(64, (b->n + 8191) / 8192));
    size_t qbytes = 0;
    uint32_t slices = 0;
    if (!noalloc_layout(uint32_t(nq), b->dp, kk, want, &qbytes, &slices))
        return set_error(HNSW_ERR_INVALID_ARGUMENT,
                         "batch too large for the no-alloc scratch: round_up(nq * 4 * round_up(dim, 32), 256) + "
                         "nq * 8 * max(1, min(k, n)) must not exceed 8 MiB");
    BruteArgs a;
    a.base = b->base.as<float>();
    a.keys = b->keys.as<uint64_t>();
    a.n = b->n;
    a.dim = b->dim;
    a.dp = b->dp;
    a.metric = b->metric;
    a.queries = d_queries;
    a.nq = uint32_t(nq);
    a.k = k;
    a.out_keys = d_keys;
    a.out_dist = d_dist;
    a.out_count = d_count;
    a.out_status = d_status;
    a.qprep = static_cast<float*>(scratch);
    a.part = reinterpret_cast<uint64_t*>(static_cast<unsigned char*>(scratch) + qbytes);
    a.tiles = slices;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : b->stream;
    CU(launch_brute_fp32(a, st), "brute kernel (no-alloc)");
    return HNSW_OK;
}

// ------------------------------------------------------------------------
// Builder and synthetic data
// ------------------------------------------------------------------------
void hnsw_params_default(uint32_t m, hnsw_params* out) {
    Params p = default_params(m);
    out->m = p.m;
    out->m0 = p.m0;
    out->ef_construction = p.ef_construction;
    out->level_multiplier = p.level_multiplier;
    out->selection = p.selection;
    out->extend_candidates = p.extend_candidates;
    out->keep_pruned = p.keep_pruned;
    out->seed = p.seed;
}

int hnsw_builder_new(size_t dim, int metric, const hnsw_params* params, hnsw_builder** out) {
    if (!out) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null output handle");
    *out = nullptr;
    if (dim == 0 || dim > kMaxDim)
        return set_error(HNSW_ERR_INVALID_DIMENSION,
                         "invalid dimension " + std::to_string(dim) + ": must be between 1 and 65536");
    if (metric < 0 || metric > 2) return set_error(HNSW_ERR_INVALID_ARGUMENT, "unknown metric");
    Params p = params ? Params{} : default_params(16);
    if (params) {
        p.m = params->m;
        p.m0 = params->m0;
        p.ef_construction = params->ef_construction;
        p.level_multiplier = params->level_multiplier;
        p.selection = params->selection ? 1 : 0;
        p.extend_candidates = params->extend_candidates != 0;
        p.keep_pruned = params->keep_pruned != 0;
        p.seed = params->seed;
    }
    const char* bad = validate_params(p);
    if (*bad) return set_error(HNSW_ERR_INVALID_PARAMETER, std::string("invalid parameter `") + bad + "`");
    auto* h = new hnsw_builder();
    h->b.reset(new Builder(uint32_t(dim), metric, p));
    *out = h;
    return HNSW_OK;
}

void hnsw_builder_free(hnsw_builder* b) { delete b; }

int hnsw_builder_insert(hnsw_builder* b, uint64_t key, const float* v, size_t dim) {
    if (!b || !v) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    if (dim != b->b->index().dim) return set_error(HNSW_ERR_DIMENSION_MISMATCH, "dimension mismatch");
    return from_err(b->b->insert(key, v));
}

int hnsw_builder_insert_batch(hnsw_builder* b, const uint64_t* keys, const float* v, size_t n, size_t dim, int threads) {
    if (!b || (n && (!keys || !v))) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    if (dim != b->b->index().dim) return set_error(HNSW_ERR_DIMENSION_MISMATCH, "dimension mismatch");
    return from_err(b->b->insert_batch(keys, v, n, threads));
}

int hnsw_builder_remove(hnsw_builder* b, uint64_t key, int* removed) {
    if (!b) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    bool r = b->b->remove(key);
    if (removed) *removed = r ? 1 : 0;
    return HNSW_OK;
}

int hnsw_builder_compact(hnsw_builder* b, int threads) {
    if (!b) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    b->b->compact(threads);
    return HNSW_OK;
}

void hnsw_gpu_build_opts_default(hnsw_gpu_build_opts* out) {
    GpuBuildOptions o;
    out->wave_fraction = o.wave_fraction;
    out->max_wave = o.max_wave;
    out->hash_cap = o.hash_cap;
    out->timing = o.timing;
}

static GpuBuildOptions build_options(const hnsw_gpu_build_opts* opts) {
    GpuBuildOptions o;
    if (opts) {
        o.wave_fraction = opts->wave_fraction;
        o.max_wave = opts->max_wave;
        o.hash_cap = opts->hash_cap;
        o.timing = opts->timing;
    }
    return o;
}

static void record_stats(hnsw_builder* b, const GpuBuildReport& r) {
    hnsw_gpu_build_stats& s = b->last;
    s.waves = r.waves;
    s.nodes = r.nodes;
    s.spills = r.spills;
    s.inexact = r.inexact;
    s.shrinks = r.shrinks;
    s.records = r.records;
    s.device_ms = r.device_ms;
    s.search_ms = r.search_ms;
    s.connect_ms = r.connect_ms;
    s.dist_search = r.dist_search;
    s.dist_select = r.dist_select;
    s.dist_connect = r.dist_connect;
    s.lists0 = r.lists0;
    s.listsU = r.listsU;
    s.search_warps_per_block = r.search_warps_per_block;
    s.search_blocks_per_sm = r.search_blocks_per_sm;
    s.connect_warps_per_block = r.connect_warps_per_block;
    s.connect_blocks_per_sm = r.connect_blocks_per_sm;
    s.hash_cap = r.hash_cap;
}

int hnsw_builder_insert_batch_gpu(hnsw_builder* b, const uint64_t* keys, const float* v, size_t n, size_t dim,
                                  int device, const hnsw_gpu_build_opts* opts) {
    if (!b || (n && (!keys || !v))) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    if (dim != b->b->index().dim) return set_error(HNSW_ERR_DIMENSION_MISMATCH, "dimension mismatch");
    const GpuBuildOptions o = build_options(opts);
    if (!(o.wave_fraction > 0.0) || o.wave_fraction > 1.0 || o.max_wave == 0)
        return set_error(HNSW_ERR_INVALID_ARGUMENT, "wave_fraction must be in (0, 1] and max_wave >= 1");
    uint32_t first = 0;
    int st = from_err(b->b->append_batch(keys, v, n, &first));
    if (st) return st;
    GpuBuildReport rep;
    st = gpu_link(b->b->graph(), first, device, o, &rep);
    if (st) {
        b->b->truncate(first);
        return st;
    }
    record_stats(b, rep);
    return HNSW_OK;
}

int hnsw_builder_compact_gpu(hnsw_builder* b, int device, const hnsw_gpu_build_opts* opts) {
    if (!b) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    const GpuBuildOptions o = build_options(opts);
    if (!(o.wave_fraction > 0.0) || o.wave_fraction > 1.0 || o.max_wave == 0)
        return set_error(HNSW_ERR_INVALID_ARGUMENT, "wave_fraction must be in (0, 1] and max_wave >= 1");
    std::unique_ptr<Builder> fresh = b->b->compacted_unlinked();
    if (!fresh) return HNSW_OK;
    GpuBuildReport rep;
    int st = gpu_link(fresh->graph(), 0, device, o, &rep);
    if (st) return st;
    if (b->b->index().quantized) fresh->enable_quantization();
    b->b = std::move(fresh);
    record_stats(b, rep);
    return HNSW_OK;
}

int hnsw_builder_gpu_stats(const hnsw_builder* b, hnsw_gpu_build_stats* out) {
    if (!b || !out) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    *out = b->last;
    return HNSW_OK;
}

int hnsw_builder_enable_quantization(hnsw_builder* b) {
    if (!b) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    b->b->enable_quantization();
    return HNSW_OK;
}

int hnsw_builder_to_bytes(const hnsw_builder* b, uint8_t** out, size_t* len) {
    if (!b || !out || !len) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    std::vector<uint8_t> bytes = write_index(b->b->index());
    auto* p = static_cast<uint8_t*>(std::malloc(std::max<size_t>(bytes.size(), 1)));
    if (!p) return set_error(HNSW_ERR_INVALID_ARGUMENT, "out of host memory");
    std::memcpy(p, bytes.data(), bytes.size());
    *out = p;
    *len = bytes.size();
    return HNSW_OK;
}

void hnsw_bytes_free(uint8_t* p) { std::free(p); }

void hnsw_synthetic_gaussian(size_t nb, size_t nq, size_t dim, uint64_t seed, float* base, float* queries) {
    synthetic_gaussian(nb, nq, dim, seed, base, queries);
}

void hnsw_synthetic_mixture(size_t nb, size_t nq, size_t dim, size_t clusters, double sigma, uint64_t seed,
                            float* base, float* queries) {
    synthetic_mixture(nb, nq, dim, clusters, sigma, seed, base, queries);
}

void hnsw_synthetic_mixture_split(size_t nb, size_t nq, size_t dim, size_t clusters, double sigma, uint64_t base_seed,
                                  uint64_t query_seed, float* base, float* queries) {
    synthetic_mixture_split(nb, nq, dim, clusters, sigma, base_seed, query_seed, base, queries);
}

}  // extern "C"
