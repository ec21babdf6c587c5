// HNSW query traversal on sm_100a: one warp per query.
//
// Restates, with identical results, HnswIndex::search_impl / search_graph /
// greedy_closest / search_layer (src/hnsw/mod.rs:460-511,
// src/hnsw/search.rs:49-161):
//   * distances in the AVX2 summation order (common.cuh), so every
//     comparison sees the reference's bits;
//   * the layer-0 beam processes each neighbor list in list order, applying
//     the visited test, the `improves` rule (strict IEEE <) and admission
//     exactly as the sequential loop does;
//   * heaps are sorted arrays ordered by (total_cmp distance, id), the
//     reference's Candidate order; the results max is the array's last entry.
// Candidates worse than the worst result once ef results exist can never be
// expanded (the loop would stop at them), so they are pruned when the
// candidate array fills; that does not change the result.
//
// Scratch per warp: the prepared query (and its int8 code), the results
// array, the candidate array, and an open-addressing visited hash over node
// ids (exact: ids are stored, not hashed away). A query that outgrows the
// warp's scratch is pushed to an overflow list and re-run by a retry kernel
// whose scratch lives in global memory (visited bitmap over all nodes).
#pragma once

#include <algorithm>

#include <cuda_bf16.h>

#include "common.cuh"
#include "device.hpp"
#include "warp_sort.cuh"

namespace hnswgpu {
namespace dev {

// Bounds checks of the checked build (-DHNSW_DEVICE_CHECKS, the
// libhnsw_gpu_checked.so target): HNSW_CHK(word, cond, site, value) is cond;
// when it fails, the first failure's site and value go to word[0], word[1]
// and the caller skips the access. In the normal build it is `true` and
// compiles away.
#ifdef HNSW_DEVICE_CHECKS
__device__ __forceinline__ bool chk_fail(uint32_t* word, uint32_t site, uint32_t value) {
    if (word && atomicCAS(word, 0u, site) == 0u) word[1] = value;
    return false;
}
#define HNSW_CHK(word, cond, site, value) ((cond) ? true : ::hnswgpu::dev::chk_fail((word), (site), uint32_t(value)))
#else
#define HNSW_CHK(word, cond, site, value) true
#endif

enum : int32_t { ST_OK = 0, ST_NON_FINITE = 3, ST_ZERO = 4, ST_QDISABLED = 7, ST_BAD_ARGUMENT = 24, ST_OVERFLOW = 25 };

struct Counters {
    uint32_t dist0 = 0, exp0 = 0, dist_up = 0, exp_up = 0;
};

// Per-warp workspace (shared memory in the fast kernel, global memory in
// the retry kernel).
struct Ws {
    float* qf;         // dp floats: prepared query
    int8_t* qc;        // dc bytes: query code
    uint4* qt;         // tensor-core traversal: the query's BF16 operands (hi, then lo)
    uint64_t* R;       // ef_cap + 1
    uint64_t* C;       // cand_cap + 1
    uint32_t* H;       // hash_cap entries, or a bitmap when bitmap_mode
    uint32_t* fr;      // 32: fresh neighbor positions
    float* fd;         // 32: distances of fresh neighbors
    // Staged gathers (null stage: off): stage_rows rows of stage_row_bytes,
    // the fresh ids in rank order, and their code norms.
    uint8_t* stage;
    uint32_t stage_rows, stage_row_bytes;
    uint32_t* fi;
    int32_t* fnorm;
    uint32_t ef_cap, cand_cap, hash_cap;
    // 16-bit tags in H (SearchGeometry::tag16): tag_sh id bits per tag,
    // tag_mask the id space.
    bool tag16;
    uint32_t tag_sh, tag_mask;
    bool bitmap_mode;  // H is a bitmap over node ids (retry kernel, or after a spill)
    uint32_t bitmap_words;
    // Persistent warps own spill areas in global memory: when the shared
    // visited hash or candidate array fills, the query continues there
    // instead of restarting. Null in the plain and retry kernels.
    uint32_t* spill_bits;   // bitmap over node ids (spill_words words, zero between queries)
    uint32_t spill_words;
    uint64_t* spill_cands;  // spill_cand_cap + 1 entries
    uint32_t spill_cand_cap;
    // The shared-memory arrays, restored after a spilled query.
    uint32_t* H0;
    uint64_t* C0;
    uint32_t cand_cap0;
    bool spilled_bits, spilled_cands;
    // Cold part of the candidate queue (retry and last-resort warps; null
    // pool in the fast kernel): an unsorted list in chunks drawn from a
    // pool. Every entry of C is below b_min, the smallest cold entry, so C's
    // head is always the best candidate; C is refilled from the cold list
    // when it runs empty, and its upper half moves there when it fills.
    uint64_t* pool;
    uint32_t* pool_next;
    uint32_t pool_chunks;
    uint32_t* tab;          // chunk ids owned by this warp (kept across its queries)
#ifdef HNSW_DEVICE_CHECKS
    uint32_t* chk;          // bounds-check word (checked build)
#endif
    uint32_t tab_cap;
    uint32_t b_chunks, b_count;
    uint64_t b_min, b_max;
};

// The bijection of the 16-bit-tag hash: x = id * kTagMul mod 2^B, inverted
// by kTagMulInv (kTagMul * kTagMulInv = 1 mod 2^32).
constexpr uint32_t kTagMul = 0x9E3779B1u;
constexpr uint32_t tag_mul_inverse(uint32_t k) {
    uint32_t x = k;
    for (int i = 0; i < 5; ++i) x *= 2u - k * x;
    return x;
}
constexpr uint32_t kTagMulInv = tag_mul_inverse(kTagMul);
static_assert(kTagMul * kTagMulInv == 1u, "tag bijection");
enum : uint32_t { VISIT_SEEN = 0, VISIT_FRESH = 1, VISIT_FULL = 2 };

// Visited test-and-set: VISIT_FRESH if id was not visited before (it is
// recorded now), VISIT_SEEN if it was, VISIT_FULL if a 16-bit-tag hash found
// no free slot within the longest probe a tag can record (id is then not in
// the set; the caller moves the set to its spill bitmap).
//
// 16-bit tags: with x = bijection(id), the home slot is x >> tag_sh and the
// tag is (x mod 2^tag_sh) << dbits | d for the probe distance d < 2^dbits - 1
// (dbits = 16 - tag_sh), so a tag never equals the empty value 0xFFFF. Slot
// s holding tag (r, d) stores the id whose x is ((s - d) << tag_sh) | r: a
// probe of id at distance d matches exactly its own tag. Slots are never
// freed during a query, so linear probing finds an id before any empty slot.
__device__ __forceinline__ uint32_t visit(Ws& w, uint32_t id) {
    if (w.bitmap_mode) {
#ifdef HNSW_DEVICE_CHECKS
        if (!HNSW_CHK(w.chk, (id >> 5) < w.bitmap_words, 1, id)) return VISIT_SEEN;
#endif
        uint32_t bit = 1u << (id & 31);
        uint32_t old = atomicOr(&w.H[id >> 5], bit);
        return (old & bit) == 0 ? VISIT_FRESH : VISIT_SEEN;
    }
    if (w.tag16) {
        const uint32_t x = (id * kTagMul) & w.tag_mask;
        const uint32_t dbits = 16u - w.tag_sh;
        const uint32_t base = (x & ((1u << w.tag_sh) - 1u)) << dbits;
        const uint32_t dlim = min((1u << dbits) - 1u, w.hash_cap);
        unsigned short* H16 = reinterpret_cast<unsigned short*>(w.H);
        uint32_t h = x >> w.tag_sh;
        for (uint32_t d = 0; d < dlim; ++d) {
            const unsigned short tag = (unsigned short)(base | d);
            const unsigned short old = atomicCAS(H16 + h, (unsigned short)0xFFFFu, tag);
            if (old == (unsigned short)0xFFFFu) return VISIT_FRESH;
            if (old == tag) return VISIT_SEEN;
            h = (h + 1u) & (w.hash_cap - 1u);
        }
        return VISIT_FULL;
    }
    // Any capacity (not only powers of two): the multiplicative hash maps
    // ids onto [0, hash_cap) and probing wraps around at the end.
    uint32_t h = uint32_t((uint64_t(id * 0x9E3779B1u) * w.hash_cap) >> 32);
    for (uint32_t probe = 0; probe < w.hash_cap; ++probe) {
        uint32_t old = atomicCAS(&w.H[h], kEmpty, id);
        if (old == kEmpty) return VISIT_FRESH;
        if (old == id) return VISIT_SEEN;
        h = h + 1 == w.hash_cap ? 0u : h + 1;
    }
    return VISIT_FRESH;  // unreachable while the load limit holds
}

// Empties the shared visited hash (all lanes).
__device__ __forceinline__ void clear_hash(Ws& w) {
    const int lane = lane_id();
    if (w.tag16) {
        uint4* h4 = reinterpret_cast<uint4*>(w.H);
        const uint4 e = make_uint4(kEmpty, kEmpty, kEmpty, kEmpty);
        for (uint32_t i = lane; i < (w.hash_cap >> 3); i += 32) h4[i] = e;
    } else {
        for (uint32_t i = lane; i < w.hash_cap; i += 32) w.H[i] = kEmpty;
    }
}

// Moves the visited set from the shared hash into the warp's spill bitmap
// (all lanes; w.spill_bits non-null) and continues in bitmap mode.
__device__ __forceinline__ void spill_visited(Ws& w) {
    const int lane = lane_id();
    if (w.tag16) {
        const unsigned short* H16 = reinterpret_cast<const unsigned short*>(w.H);
        const uint32_t dbits = 16u - w.tag_sh, dmask = (1u << dbits) - 1u;
        for (uint32_t i = lane; i < w.hash_cap; i += 32) {
            const uint32_t t = H16[i];
            if (t == 0xFFFFu) continue;
            const uint32_t home = (i - (t & dmask)) & (w.hash_cap - 1u);
            const uint32_t v = (((home << w.tag_sh) | (t >> dbits)) * kTagMulInv) & w.tag_mask;
            atomicOr(&w.spill_bits[v >> 5], 1u << (v & 31));
        }
    } else {
        for (uint32_t i = lane; i < w.hash_cap; i += 32) {
            const uint32_t v = w.H[i];
            if (v != kEmpty) atomicOr(&w.spill_bits[v >> 5], 1u << (v & 31));
        }
    }
    __syncwarp();
    w.H = w.spill_bits;
    w.bitmap_mode = true;
    w.bitmap_words = w.spill_words;
    w.spilled_bits = true;
}

// Visited test of one neighbor list chunk (every lane, `valid` lanes hold
// ids). A tag hash that cannot place an id moves the set to the spill
// bitmap, where the id is then recorded; without a spill area the query
// goes to the retry pass (*retry).
__device__ __forceinline__ bool visit_chunk(Ws& w, uint32_t id, bool valid, bool* retry) {
    uint32_t vr = valid ? visit(w, id) : VISIT_SEEN;
    if (w.tag16 && !w.bitmap_mode && __any_sync(kFull, vr == VISIT_FULL)) {
        if (!w.spill_bits) {
            *retry = true;
            return false;
        }
        spill_visited(w);
        if (vr == VISIT_FULL) {
            atomicOr(&w.H[id >> 5], 1u << (id & 31));
            vr = VISIT_FRESH;
        }
        __syncwarp();
    }
    return vr == VISIT_FRESH;
}

struct QueryCtx {
    const SearchArgs* a;
    Ws* w;
    uint32_t qi;
    int metric;
    bool quant;
    float s2;
    int qnorm;  // squared norm of the query code (L2 on codes)
    float qn2;  // squared f32 norm of the prepared query (tensor-core L2)
    bool use_filter;
    bool by_node;
    const uint64_t* fbits;
    uint64_t fnbits;
    Counters cnt;
};

__device__ __forceinline__ bool admit(const QueryCtx& c, uint32_t id) {
    const DeviceIndexView& ix = c.a->ix;
    if (ix.has_dead && ((__ldg(ix.dead + (id >> 5)) >> (id & 31)) & 1u)) return false;
    if (!c.use_filter) return true;
    uint64_t key = (ix.keys_are_ids || c.by_node) ? uint64_t(id) : __ldg(ix.keys + id);
    return key < c.fnbits && ((__ldg(c.fbits + (key >> 6)) >> (key & 63)) & 1ull);
}

// Distance kinds a kernel is built for. DK_ANY decides per query at run time
// (f32 rows or int8 codes, any metric, rows loaded directly or staged);
// DK_L2 and DK_DOT are f32 rows loaded directly with the L2 sum or the dot
// sum (inner product, cosine), so the kernel carries one distance loop
// instead of all of them: less code in the traversal loop to fetch.
// DK_TC1 and DK_TC3 compute the distances of each neighbor list on the
// tensor cores (BF16, or the 3-term hi/lo split) for the tensor-core
// traversal; the results are re-ranked with exact f32 distances.
constexpr int DK_ANY = 0, DK_L2 = 1, DK_DOT = 2, DK_TC1 = 3, DK_TC3 = 4;
__host__ __device__ constexpr bool is_tc(int dk) { return dk == DK_TC1 || dk == DK_TC3; }

// Position (in BF16 values) of dimension d in a tensor-core row: within each
// block of 32 values, lane t of an mma quad reads one 16-byte word holding
// k = 2t, 2t+1, 2t+8, 2t+9 of the block's first 16 dimensions, then the
// same of its second 16 (the A/B fragment order of mma.m16n8k16).
__host__ __device__ __forceinline__ uint32_t tc_row_pos(uint32_t d) {
    const uint32_t o = d & 31u, kb = o >> 4, r = o & 15u;
    return (d & ~31u) + 8u * ((r & 7u) >> 1) + 4u * kb + 2u * (r >> 3) + (r & 1u);
}

// D += A.B for one m16n8k16 tile: BF16 operands, FP32 accumulation.
__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                               uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Distances of the neighbors at the list positions in F (lane p holds the
// id at position p) on the tensor cores, into w.fd[p]. The 32 positions are
// the rows of two 16-row A tiles and the query is every column of B, so one
// m16n8k16 per 16 dimensions and tile. Lane (g, t) = (lane / 4, lane % 4)
// loads positions g, g+8, g+16, g+24, one 16-byte word per 32 dimensions of
// each (tc_row_pos); the dot of position p ends in lane 4 (p % 8) + p / 8.
// X3 adds x_hi.q_lo and x_lo.q_hi to x_hi.q_hi. L2 uses |q|^2 + |x|^2 - 2 q.x.
template <bool X3>
__device__ __forceinline__ void tc_chunk_distances(QueryCtx& c, uint32_t my_id, uint32_t F) {
    const DeviceIndexView& ix = c.a->ix;
    Ws& w = *c.w;
    const int lane = lane_id();
    const int g = lane >> 2, t = lane & 3;
    const uint32_t stride = ix.dt >> 3, blocks = ix.dt >> 5;
    const uint4 z = make_uint4(0u, 0u, 0u, 0u);
    size_t off[4];
    bool on[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const uint32_t id = __shfl_sync(kFull, my_id, g + 8 * j);
        on[j] = (F >> (g + 8 * j)) & 1u;
        off[j] = size_t(on[j] ? id : 0u) * stride + uint32_t(t);
    }
    float acc0[4] = {0.f, 0.f, 0.f, 0.f}, acc1[4] = {0.f, 0.f, 0.f, 0.f};
    for (uint32_t b = 0; b < blocks; ++b) {
        uint4 x[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) x[j] = on[j] ? __ldg(ix.tc_hi + off[j] + 4u * b) : z;
        const uint4 q = w.qt[4u * b + uint32_t(t)];
        mma_bf16_16816(acc0, x[0].x, x[1].x, x[0].y, x[1].y, q.x, q.y);
        mma_bf16_16816(acc1, x[2].x, x[3].x, x[2].y, x[3].y, q.x, q.y);
        mma_bf16_16816(acc0, x[0].z, x[1].z, x[0].w, x[1].w, q.z, q.w);
        mma_bf16_16816(acc1, x[2].z, x[3].z, x[2].w, x[3].w, q.z, q.w);
        if constexpr (X3) {
            const uint4 ql = w.qt[stride + 4u * b + uint32_t(t)];
            mma_bf16_16816(acc0, x[0].x, x[1].x, x[0].y, x[1].y, ql.x, ql.y);
            mma_bf16_16816(acc1, x[2].x, x[3].x, x[2].y, x[3].y, ql.x, ql.y);
            mma_bf16_16816(acc0, x[0].z, x[1].z, x[0].w, x[1].w, ql.z, ql.w);
            mma_bf16_16816(acc1, x[2].z, x[3].z, x[2].w, x[3].w, ql.z, ql.w);
            uint4 y[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) y[j] = on[j] ? __ldg(ix.tc_lo + off[j] + 4u * b) : z;
            mma_bf16_16816(acc0, y[0].x, y[1].x, y[0].y, y[1].y, q.x, q.y);
            mma_bf16_16816(acc1, y[2].x, y[3].x, y[2].y, y[3].y, q.x, q.y);
            mma_bf16_16816(acc0, y[0].z, y[1].z, y[0].w, y[1].w, q.z, q.w);
            mma_bf16_16816(acc1, y[2].z, y[3].z, y[2].w, y[3].w, q.z, q.w);
        }
    }
    // acc0[0] / acc0[2]: positions g / g+8; acc1[0] / acc1[2]: g+16 / g+24.
    const float v = t == 0 ? acc0[0] : t == 1 ? acc0[2] : t == 2 ? acc1[0] : acc1[2];
    const float dot = __shfl_sync(kFull, v, 4 * (lane & 7) + (lane >> 3));
    if ((F >> lane) & 1u) {
        float d;
        if (c.metric == 0) d = c.qn2 + __ldg(ix.xnorm + my_id) - 2.0f * dot;
        else d = metric_from_sum(c.metric, dot);
        w.fd[lane] = d;
    }
    __syncwarp();
}

// The query's BF16 operands (hi, and for X3 lo = bf16(q - hi)) in the
// tensor-core row order, and its squared norm; all lanes call after prepare.
template <bool X3>
__device__ __forceinline__ void tc_prepare_query(QueryCtx& c) {
    const DeviceIndexView& ix = c.a->ix;
    Ws& w = *c.w;
    const int lane = lane_id();
    __nv_bfloat16* hi = reinterpret_cast<__nv_bfloat16*>(w.qt);
    __nv_bfloat16* lo = hi + ix.dt;
    float sq = 0.0f;
    for (uint32_t d = lane; d < ix.dt; d += 32) {
        const float x = d < ix.dim ? w.qf[d] : 0.0f;
        const __nv_bfloat16 h = __float2bfloat16_rn(x);
        hi[tc_row_pos(d)] = h;
        if (X3) lo[tc_row_pos(d)] = __float2bfloat16_rn(__fsub_rn(x, __bfloat162float(h)));
        sq = __fadd_rn(sq, __fmul_rn(x, x));
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) sq = __fadd_rn(sq, __shfl_xor_sync(kFull, sq, off));
    c.qn2 = sq;
    __syncwarp();
}

// Distance from the query to node `id` for the group of 8 lanes (valid in
// every lane of the group). All 32 lanes call; `id` may differ per group.
template <int DK = DK_ANY>
__device__ __forceinline__ float group_distance(const QueryCtx& c, uint32_t id, int g8) {
    const DeviceIndexView& ix = c.a->ix;
    if (DK == DK_ANY && c.quant) {
        int dot = group_i8dot(ix.codes + size_t(id) * ix.dc, c.w->qc, int(ix.dc), g8);
        long long l2 = 0;
        if (c.metric == 0) l2 = (long long)c.qnorm + (long long)__ldg(ix.code_norm + id) - 2ll * (long long)dot;
        return sq_distance(c.metric, dot, l2, c.s2);
    }
    const float* row = ix.vec + size_t(id) * ix.dp;
    const bool l2 = DK == DK_ANY ? c.metric == 0 : DK == DK_L2;
    float s = l2 ? group_sum<true>(row, c.w->qf, int(ix.dim), g8) : group_sum<false>(row, c.w->qf, int(ix.dim), g8);
    s = __shfl_sync(kFull, s, (lane_id() & ~7));
    return metric_from_sum(c.metric, s);
}

// group_distance for a row staged in shared memory (`norm`: its code norm).
__device__ __forceinline__ float staged_distance(const QueryCtx& c, const uint8_t* row, int32_t norm, int g8) {
    const DeviceIndexView& ix = c.a->ix;
    if (c.quant) {
        int dot = group_i8dot<true>(reinterpret_cast<const int8_t*>(row), c.w->qc, int(ix.dc), g8);
        long long l2 = 0;
        if (c.metric == 0) l2 = (long long)c.qnorm + (long long)norm - 2ll * (long long)dot;
        return sq_distance(c.metric, dot, l2, c.s2);
    }
    const float* r = reinterpret_cast<const float*>(row);
    float s = c.metric == 0 ? group_sum<true, true>(r, c.w->qf, int(ix.dim), g8)
                            : group_sum<false, true>(r, c.w->qf, int(ix.dim), g8);
    s = __shfl_sync(kFull, s, (lane_id() & ~7));
    return metric_from_sum(c.metric, s);
}

// Exact f32 distance (for the re-rank), valid in every lane of the group.
__device__ __forceinline__ float group_exact(const QueryCtx& c, uint32_t id, int g8) {
    const DeviceIndexView& ix = c.a->ix;
    const float* row = ix.vec + size_t(id) * ix.dp;
    float s = c.metric == 0 ? group_sum<true>(row, c.w->qf, int(ix.dim), g8)
                            : group_sum<false>(row, c.w->qf, int(ix.dim), g8);
    s = __shfl_sync(kFull, s, (lane_id() & ~7));
    return metric_from_sum(c.metric, s);
}

// Computes distances for the neighbors at positions fr[0..nf) of the
// current chunk (ids in lane order `ids`), writing fd[pos].
template <int DK = DK_ANY>
__device__ __forceinline__ void chunk_distances(QueryCtx& c, uint32_t my_id, uint32_t F) {
    Ws& w = *c.w;
    const int lane = lane_id();
    const int g = lane >> 3, g8 = lane & 7;
    if constexpr (is_tc(DK)) {
        tc_chunk_distances<DK == DK_TC3>(c, my_id, F);
        return;
    }
    const bool stage = DK == DK_ANY && w.stage != nullptr;
    // Ranks of fresh lanes -> compact list of positions.
    if ((F >> lane) & 1u) {
        const uint32_t rk = __popc(F & ((1u << lane) - 1u));
        w.fr[rk] = uint32_t(lane);
        if (stage) w.fi[rk] = my_id;
    }
    __syncwarp();
    const uint32_t nf = __popc(F);
    if (stage) {
        // All rows of a round in flight at once, one wait, then the
        // distances from shared memory.
        const DeviceIndexView& ix = c.a->ix;
        const uint32_t rb = w.stage_row_bytes, cpr = rb >> 4;
        const char* src = c.quant ? reinterpret_cast<const char*>(ix.codes) : reinterpret_cast<const char*>(ix.vec);
        const size_t stride = c.quant ? size_t(ix.dc) : size_t(ix.dp) * 4;
        const bool norms = c.quant && c.metric == 0;
        for (uint32_t r0 = 0; r0 < nf; r0 += w.stage_rows) {
            const uint32_t nr = min(w.stage_rows, nf - r0);
            for (uint32_t t = lane; t < nr * cpr; t += 32) {
                const uint32_t slot = t / cpr, part = t - slot * cpr;
                cp_async16(w.stage + slot * rb + part * 16, src + size_t(w.fi[r0 + slot]) * stride + part * 16);
            }
            if (norms && uint32_t(lane) < nr) cp_async4(w.fnorm + lane, ix.code_norm + w.fi[r0 + lane]);
            cp_async_wait_all();
            __syncwarp();
            for (uint32_t s0 = 0; s0 < nr; s0 += 4) {
                const uint32_t slot = s0 + uint32_t(g);
                const bool active = slot < nr;
                const uint32_t sl = active ? slot : 0u;
                const float d = staged_distance(c, w.stage + sl * rb, norms ? w.fnorm[sl] : 0, g8);
                if (active && g8 == 0) w.fd[w.fr[r0 + slot]] = d;
            }
            __syncwarp();
        }
        return;
    }
    if (DK != DK_ANY || !c.quant) {
        // f32 rows: two rows per group while at least five remain.
        const DeviceIndexView& ix = c.a->ix;
        const bool l2 = DK == DK_ANY ? c.metric == 0 : DK == DK_L2;
        uint32_t r = 0;
        for (; r + 4 < nf; r += 8) {
            const uint32_t sa = r + uint32_t(g), sb = r + 4 + uint32_t(g);
            const bool aa = sa < nf, ab = sb < nf;
            const uint32_t pa = aa ? w.fr[sa] : w.fr[0], pb = ab ? w.fr[sb] : w.fr[0];
            const uint32_t ida = __shfl_sync(kFull, my_id, int(pa)), idb = __shfl_sync(kFull, my_id, int(pb));
            float s0, s1;
            if (l2)
                group_sum2<true>(ix.vec + size_t(ida) * ix.dp, ix.vec + size_t(idb) * ix.dp, w.qf, int(ix.dim), g8, s0,
                                 s1);
            else
                group_sum2<false>(ix.vec + size_t(ida) * ix.dp, ix.vec + size_t(idb) * ix.dp, w.qf, int(ix.dim), g8,
                                  s0, s1);
            s0 = __shfl_sync(kFull, s0, (lane & ~7));
            s1 = __shfl_sync(kFull, s1, (lane & ~7));
            if (aa && g8 == 0) w.fd[pa] = metric_from_sum(c.metric, s0);
            if (ab && g8 == 0) w.fd[pb] = metric_from_sum(c.metric, s1);
        }
        if (r < nf) {
            const uint32_t slot = r + uint32_t(g);
            const bool active = slot < nf;
            const uint32_t pos = active ? w.fr[slot] : w.fr[0];
            const uint32_t id = __shfl_sync(kFull, my_id, int(pos));
            const float d = group_distance<DK>(c, id, g8);
            if (active && g8 == 0) w.fd[pos] = d;
        }
        __syncwarp();
        return;
    }
    if constexpr (DK == DK_ANY) {
        // int8 codes, one row per group.
        for (uint32_t r = 0; r < nf; r += 4) {
            uint32_t slot = r + uint32_t(g);
            bool active = slot < nf;
            uint32_t pos = active ? w.fr[slot] : w.fr[0];
            uint32_t id = __shfl_sync(kFull, my_id, int(pos));
            float d = group_distance(c, id, g8);
            if (active && g8 == 0) w.fd[pos] = d;
        }
        __syncwarp();
    }
}

// greedy_closest (src/hnsw/search.rs:49-68) on an upper layer.
template <int DK = DK_ANY>
__device__ __forceinline__ uint64_t greedy_layer(QueryCtx& c, uint64_t best, uint32_t layer) {
    const DeviceIndexView& ix = c.a->ix;
    Ws& w = *c.w;
    const int lane = lane_id();
    for (;;) {
        const uint32_t from = pid(best);
#ifdef HNSW_DEVICE_CHECKS
        if (!HNSW_CHK(w.chk, from < ix.n, 4, from)) return best;
#endif
        const uint32_t* blk = ix.adjU + size_t(__ldg(ix.up_off + from) + (layer - 1)) * ix.mp;
        c.cnt.exp_up++;
        float bd = pdist(best);
        uint32_t bid = from;
        for (uint32_t base = 0; base < ix.m; base += 32) {
            uint32_t id = (base + lane < ix.m) ? __ldg(blk + base + lane) : kEmpty;
#ifdef HNSW_DEVICE_CHECKS
            if (!HNSW_CHK(w.chk, id == kEmpty || id < ix.n, 2, id)) id = kEmpty;
#endif
            uint32_t V = __ballot_sync(kFull, id != kEmpty);
            if (V == 0) break;
            chunk_distances<DK>(c, id, V);
            c.cnt.dist_up += __popc(V);
            // First strict minimum in list order (IEEE comparison, as d < best.distance).
            float d = ((V >> lane) & 1u) ? w.fd[lane] : __int_as_float(0x7f800000);
            int idx = lane;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                float od = __shfl_down_sync(kFull, d, off);
                int oi = __shfl_down_sync(kFull, idx, off);
                if (od < d || (od == d && oi < idx)) {
                    d = od;
                    idx = oi;
                }
            }
            d = __shfl_sync(kFull, d, 0);
            idx = __shfl_sync(kFull, idx, 0);
            if (((V >> idx) & 1u) && d < bd) {
                bd = d;
                bid = __shfl_sync(kFull, id, idx);
            }
            if (V != kFull) break;
        }
        if (bid == from) return best;
        best = (uint64_t(fkey(bd)) << 32) | bid;
    }
}

// Lane of the r-th (from 0) set bit of m; m has more than r bits set.
__device__ __forceinline__ int nth_set(uint32_t m, int r) {
    for (int i = 0; i < r; ++i) m &= m - 1u;
    return __ffs(int(m)) - 1;
}

__device__ __forceinline__ uint64_t* cold_slot(const Ws& w, uint32_t pos) {
#ifdef HNSW_DEVICE_CHECKS
    if (!HNSW_CHK(w.chk, (pos >> kColdChunkShift) < w.b_chunks, 7, pos) ||
        !HNSW_CHK(w.chk, w.tab[pos >> kColdChunkShift] < w.pool_chunks, 8, w.tab[pos >> kColdChunkShift]))
        return w.pool;
#endif
    return w.pool + (size_t(w.tab[pos >> kColdChunkShift]) << kColdChunkShift) + (pos & (kColdChunk - 1));
}

__device__ __forceinline__ void cold_reset(Ws& w) {
    w.b_count = 0;
    w.b_min = ~0ull;
    w.b_max = 0;
}

// Appends the entries x of the lanes in S to the cold list. Returns false
// when the pool has no chunk left. All lanes call.
static __device__ bool cold_append(Ws& w, uint32_t S, uint64_t x) {
    const int lane = lane_id();
    const uint32_t n = __popc(S);
    if (n == 0) return true;
    if (w.b_count + n > (w.b_chunks << kColdChunkShift)) {
        if (w.b_chunks >= w.tab_cap) return false;
        uint32_t c = 0;
        if (lane == 0) c = atomicAdd(w.pool_next, 1u);
        c = __shfl_sync(kFull, c, 0);
        if (c >= w.pool_chunks) return false;
        if (lane == 0) w.tab[w.b_chunks] = c;
        ++w.b_chunks;
        __syncwarp();
    }
    const bool in = (S >> lane) & 1u;
    if (in) *cold_slot(w, w.b_count + __popc(S & ((1u << lane) - 1u))) = x;
    w.b_count += n;
    w.b_min = min(w.b_min, warp_min_u64(in ? x : ~0ull));
    w.b_max = max(w.b_max, warp_max_u64(in ? x : 0ull));
    __syncwarp();
    return true;
}

// Makes room for `need` more candidates: compacts the queue to the front,
// then drops candidates worse than the worst of ef results (they can never be
// expanded), then moves the upper part of the array to the cold list.
// Returns false if the queue is still too small.
template <bool COLD>
__device__ __forceinline__ bool make_room(Ws& w, uint32_t& head, uint32_t& tail, uint32_t need, uint32_t rs,
                                          uint32_t ef) {
    if (tail + need <= w.cand_cap) return true;
    const int lane = lane_id();
    if (head > 0) {
        const uint32_t n = tail - head;
        for (uint32_t b = 0; b < n; b += 32) {
            const uint32_t j = b + lane;
            const uint64_t v = j < n ? w.C[head + j] : 0;
            __syncwarp();
            if (j < n) w.C[j] = v;
            __syncwarp();
        }
        head = 0;
        tail = n;
    }
    if (tail + need > w.cand_cap && rs >= ef) {
        const float wd = pdist(w.R[rs - 1]);
        uint32_t keep = head;
        for (uint32_t b = head; b < tail; b += 32) {
            const uint32_t j = b + lane;
            const bool ok = j < tail && !(pdist(w.C[j]) > wd);
            keep += __popc(__ballot_sync(kFull, ok));
        }
        tail = keep;
    }
    if (tail + need > w.cand_cap && w.spill_cands && !w.spilled_cands && w.spill_cand_cap > w.cand_cap) {
        // Move the queue to the warp's larger global array.
        const uint32_t n = tail - head;
        for (uint32_t b = 0; b < n; b += 32) {
            const uint32_t j = b + lane;
            if (j < n) w.spill_cands[j] = w.C[head + j];
        }
        __syncwarp();
        w.C = w.spill_cands;
        w.cand_cap = w.spill_cand_cap;
        w.spilled_cands = true;
        head = 0;
        tail = n;
    }
    if (COLD && tail + need > w.cand_cap && w.pool && need <= w.cand_cap) {
        // Keep the lower half (or less, to fit `need`); the rest is larger
        // than everything kept, so the cold list's minimum stays above C.
        const uint32_t keep = min((tail - head) >> 1, w.cand_cap - need);
        for (uint32_t b = head + keep; b < tail; b += 32) {
            const uint32_t j = b + lane;
            const bool in = j < tail;
            const uint64_t v = in ? w.C[j] : 0;
            if (!cold_append(w, __ballot_sync(kFull, in), v)) return false;
        }
        tail = head + keep;
    }
    return tail + need <= w.cand_cap;
}

// Loads cold entries b + lane + 32k, k = 0..3 (b a multiple of 128, so the
// four lie in one chunk): four independent loads in flight per lane.
__device__ __forceinline__ void cold_load4(const Ws& w, uint32_t b, uint64_t (&v)[4], bool (&ok)[4]) {
    const int lane = lane_id();
    const uint64_t* base =
        w.pool + (size_t(w.tab[b >> kColdChunkShift]) << kColdChunkShift) + (b & (kColdChunk - 1));
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        ok[k] = b + uint32_t(lane + 32 * k) < w.b_count;
        v[k] = ok[k] ? base[lane + 32 * k] : 0ull;
    }
}

// Refills the empty candidate array from the cold list with its smallest
// entries, in order (at least one, at most half the array). When ef results
// exist (`full`), cold entries worse than the worst result are dropped
// first: they can never be expanded. The 64 words at w.fr serve as the
// histogram of a radix selection of the cut.
static __device__ void cold_refill(Ws& w, uint32_t& head, uint32_t& tail, bool full, float worst) {
    const int lane = lane_id();
    const uint32_t lt = (1u << lane) - 1u;
    head = tail = 0;
    if (full) {
        uint32_t keep = 0;
        uint64_t mn = ~0ull, mx = 0;
        for (uint32_t b = 0; b < w.b_count; b += 128) {
            uint64_t v[4];
            bool ok[4];
            cold_load4(w, b, v, ok);
            __syncwarp();
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const bool kp = ok[k] && !(pdist(v[k]) > worst);
                const uint32_t K = __ballot_sync(kFull, kp);
                if (kp) {
                    *cold_slot(w, keep + __popc(K & lt)) = v[k];
                    mn = min(mn, v[k]);
                    mx = max(mx, v[k]);
                }
                keep += __popc(K);
            }
            __syncwarp();
        }
        w.b_count = keep;
        w.b_min = warp_min_u64(mn);
        w.b_max = warp_max_u64(mx);
        if (keep == 0) return;
    }
    const uint32_t target = max(1u, min(w.b_count, w.cand_cap >> 1));
    // Take every cold entry below `bound`. Entries are distinct, and b_max
    // is below ~0 (ids are below the sentinel), so bound = b_max + 1 takes all.
    uint64_t bound = w.b_max + 1;
    if (w.b_count > target) {
        // Window [lo, lo + 2^wbits) holding the undecided entries, split into
        // 64 bins of 2^s keys; `known` entries lie below the window.
        const int p = 63 - __clzll(static_cast<long long>(w.b_min ^ w.b_max));
        int wbits = p + 1;
        int s = max(wbits - 6, 0);
        uint64_t lo = wbits >= 64 ? 0ull : (w.b_min & ~((1ull << wbits) - 1ull));
        uint32_t known = 0;
        uint32_t* hist = w.fr;
        for (int pass = 0; pass < 12; ++pass) {
            hist[lane] = 0;
            hist[lane + 32] = 0;
            __syncwarp();
            for (uint32_t b = 0; b < w.b_count; b += 128) {
                uint64_t v[4];
                bool ok[4];
                cold_load4(w, b, v, ok);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const uint64_t off = v[k] - lo;
                    if (ok[k] && v[k] >= lo && (wbits >= 64 || (off >> wbits) == 0))
                        atomicAdd(&hist[uint32_t(off >> s)], 1u);
                }
            }
            __syncwarp();
            const uint32_t c0 = hist[2 * lane], c1 = hist[2 * lane + 1];
            uint32_t incl = c0 + c1;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t o = __shfl_up_sync(kFull, incl, off);
                if (lane >= off) incl += o;
            }
            const uint32_t excl = incl - c0 - c1;
            // Largest bin count j with known + (entries in bins below j) <= target.
            const bool q1 = known + excl + c0 <= target, q2 = known + incl <= target;
            const uint32_t jstar = __reduce_add_sync(kFull, uint32_t(q1) + uint32_t(q2));
            const uint32_t taken =
                known + __reduce_max_sync(kFull, q2 ? incl : (q1 ? excl + c0 : 0u));
            __syncwarp();
            bound = lo + (uint64_t(jstar) << s);
            if ((taken >= 1 && 2 * taken >= target) || s == 0) break;
            known = taken;
            lo += uint64_t(jstar) << s;
            wbits = s;
            s = max(s - 6, 0);
        }
    }
    // Move the entries below `bound` into C through a 32-entry stage held one
    // per lane; compact the others in place.
    uint64_t stage = 0, mn = ~0ull, mx = 0;
    uint32_t sn = 0, keep = 0;
    for (uint32_t b = 0; b < w.b_count; b += 128) {
        uint64_t vv[4];
        bool okv[4];
        cold_load4(w, b, vv, okv);
        __syncwarp();
#pragma unroll 1
        for (int k = 0; k < 4; ++k) {
            const uint64_t v = vv[k];
            const bool valid = okv[k];
            const bool sel = valid && v < bound, kp = valid && !sel;
            const uint32_t S = __ballot_sync(kFull, sel), K = __ballot_sync(kFull, kp);
            if (kp) {
                *cold_slot(w, keep + __popc(K & lt)) = v;
                mn = min(mn, v);
                mx = max(mx, v);
            }
            keep += __popc(K);
            const uint32_t ns = __popc(S);
            if (ns) {
                // Lanes sn.. receive the selected entries in lane order.
                const int r = lane - int(sn);
                const bool take = r >= 0 && r < int(ns);
                const uint64_t got = __shfl_sync(kFull, v, take ? nth_set(S, r) : 0);
                if (take) stage = got;
                const uint32_t fit = min(ns, 32u - sn);
                sn += fit;
                if (sn == 32) {
                    batch_merge(w.C, 0, tail, kFull, stage, w.cand_cap);
                    tail += 32;
                    const uint32_t r2 = uint32_t(lane) + fit;
                    const uint64_t rest = __shfl_sync(kFull, v, r2 < ns ? nth_set(S, int(r2)) : 0);
                    if (r2 < ns) stage = rest;
                    sn = ns - fit;
                }
            }
        }
        __syncwarp();
    }
    if (sn) {
        batch_merge(w.C, 0, tail, (sn == 32 ? kFull : ((1u << sn) - 1u)), stage, w.cand_cap);
        tail += sn;
    }
    __syncwarp();
    w.b_count = keep;
    w.b_min = warp_min_u64(mn);
    w.b_max = warp_max_u64(mx);
}

// search_layer on layer 0 (src/hnsw/search.rs:81-142). Returns the number of
// results in w.R (sorted ascending), or -1 on scratch overflow.
// COLD: the cold list is compiled in (retry kernels, and the fast kernel's
// variant for batches whose queues outgrow shared memory, e.g. selective
// filters); without it the hot loop keeps fewer registers live.
template <bool COLD, int DK = DK_ANY>
__device__ __forceinline__ int layer0(QueryCtx& c, uint64_t ep, uint32_t ef) {
    const DeviceIndexView& ix = c.a->ix;
    Ws& w = *c.w;
    const int lane = lane_id();
    // Reset the visited set (a spill bitmap is cleared when its query ends).
    if (w.bitmap_mode) {
        for (uint32_t i = lane; i < w.bitmap_words; i += 32) w.H[i] = 0;
    } else {
        clear_hash(w);
    }
    __syncwarp();
    const uint32_t hash_limit = (w.hash_cap >> 2) * 3;
    uint32_t visited = 0;
    uint32_t rs = 0, head = 0, tail = 0;
    cold_reset(w);
    if (lane == 0) visit(w, pid(ep));
    visited = 1;
    if (lane == 0) w.C[0] = ep;
    tail = 1;
    if (admit(c, pid(ep))) {
        if (lane == 0) w.R[0] = ep;
        rs = 1;
    }
    __syncwarp();
    for (;;) {
        if (head == tail) {
            if (!COLD || w.b_count == 0) break;
            cold_refill(w, head, tail, rs >= ef, rs > 0 ? pdist(w.R[rs - 1]) : 0.0f);
            if (head == tail) break;
        }
        const uint64_t cur = w.C[head];
        ++head;
        const float worst0 = rs > 0 ? pdist(w.R[rs - 1]) : 0.0f;
        if (rs >= ef && pdist(cur) > worst0) break;
        c.cnt.exp0++;
#ifdef HNSW_DEVICE_CHECKS
        if (!HNSW_CHK(w.chk, pid(cur) < ix.n, 3, pid(cur))) return -1;
#endif
        const uint32_t* row = ix.adj0 + size_t(pid(cur)) * ix.m0p;
        // The next candidate in the queue is usually the next expansion.
        if (lane == 0 && head < tail) prefetch_l2(ix.adj0 + size_t(pid(w.C[head])) * ix.m0p, ix.m0p * 4);
        for (uint32_t base = 0; base < ix.m0; base += 32) {
#ifdef HNSW_DEVICE_CHECKS
            uint32_t id = (base + lane < ix.m0) ? __ldg(row + base + lane) : kEmpty;
            if (!HNSW_CHK(w.chk, id == kEmpty || id < ix.n, 2, id)) id = kEmpty;
#else
            uint32_t id = (base + lane < ix.m0) ? __ldg(row + base + lane) : kEmpty;
#endif
            const bool valid = id != kEmpty;
            const uint32_t V = __ballot_sync(kFull, valid);
            if (V == 0) break;
            if (!w.bitmap_mode && visited + __popc(V) > hash_limit) {
                if (!w.spill_bits) return -1;
                // Move the visited set into the warp's global bitmap.
                spill_visited(w);
            }
            bool retry = false;
            const bool fresh = visit_chunk(w, id, valid, &retry);
            if (retry) return -1;
            if (is_tc(DK)) {
                if (fresh) {
                    prefetch_l2(ix.tc_hi + size_t(id) * (ix.dt >> 3), ix.dt * 2);
                    if (DK == DK_TC3) prefetch_l2(ix.tc_lo + size_t(id) * (ix.dt >> 3), ix.dt * 2);
                }
            } else if (fresh && !w.stage) {
                if (c.quant) prefetch_l2(ix.codes + size_t(id) * ix.dc, ix.dc);
                else prefetch_l2(ix.vec + size_t(id) * ix.dp, ix.dp * 4);
            }
            const uint32_t F = __ballot_sync(kFull, fresh);
            visited += __popc(F);
            if (F != 0) {
                chunk_distances<DK>(c, id, F);
                c.cnt.dist0 += __popc(F);
                const bool adm = fresh && admit(c, id);
                const uint32_t A = __ballot_sync(kFull, adm);
                float my_d = fresh ? w.fd[lane] : 0.0f;
                uint32_t P = F;
                if (rs >= ef) {
                    float wd = pdist(w.R[rs - 1]);
                    P &= __ballot_sync(kFull, fresh && my_d < wd);
                }
                if (P == 0) {
                    if (V != kFull) break;
                    continue;
                }
                const bool inP = (P >> lane) & 1u;
                const uint64_t my_x = pack(my_d, id);
                // Equal distances (IEEE, so -0 == +0) among the improving
                // neighbors, or with a current result, make the order of
                // evaluation matter: take the sequential path for this list.
                const float dz = __fadd_rn(my_d, 0.0f);
                const unsigned same =
                    __match_any_sync(kFull, inP ? __float_as_uint(dz) : (0x7FC00000u | uint32_t(lane)));
                uint32_t pr = 0;  // results below my_x
                bool tie = inP && __popc(same) > 1;
                if (inP) {
                    pr = lower_bound(w.R, 0, rs, my_x);
                    if (pr < rs && pdist(w.R[pr]) == my_d) tie = true;
                    if (pr > 0 && pdist(w.R[pr - 1]) == my_d) tie = true;
                }
                if (!__any_sync(kFull, tie)) {
                    // Rank of each neighbor among the results and the admitted
                    // neighbors before it in list order; it improves iff the
                    // rank is below ef (src/hnsw/search.rs:125).
                    uint32_t before = 0;
                    for (uint32_t bits = A & P; bits; bits &= bits - 1) {
                        const int j = __ffs(bits) - 1;
                        const uint64_t xj = __shfl_sync(kFull, my_x, j);
                        before += (j < lane && xj < my_x) ? 1u : 0u;
                    }
                    const uint32_t I = __ballot_sync(kFull, inP && pr + before < ef);
                    const uint32_t IR = I & A;
                    if (IR) {
                        // fr/fd (dead until the next chunk's distances) hold
                        // the merges' new entries.
                        batch_merge_gather(w.R, 0, rs, IR, my_x, ef, reinterpret_cast<uint64_t*>(w.fr));
                        rs = min(rs + uint32_t(__popc(IR)), ef);
                    }
                    if (I) {
                        // Entries above the cold minimum join the cold list.
                        uint32_t IA = I, IB = 0;
                        if (COLD && w.b_count) {
                            IB = I & __ballot_sync(kFull, my_x > w.b_min);
                            IA &= ~IB;
                        }
                        if (IA) {
                            if (!make_room<COLD>(w, head, tail, uint32_t(__popc(IA)), rs, ef)) return -1;
                            if (COLD && w.b_count) {
                                const uint32_t mv = IA & __ballot_sync(kFull, my_x > w.b_min);
                                IA &= ~mv;
                                IB |= mv;
                            }
                            if (IA) {
                                batch_merge_gather(w.C, head, tail, IA, my_x, w.cand_cap,
                                                   reinterpret_cast<uint64_t*>(w.fr));
                                tail += uint32_t(__popc(IA));
                            }
                        }
                        if (COLD && IB && !cold_append(w, IB, my_x)) return -1;
                    }
                } else {
                    while (P) {
                        const int i = __ffs(P) - 1;
                        P &= P - 1;
                        const float d = __shfl_sync(kFull, my_d, i);
                        const uint32_t nid = __shfl_sync(kFull, id, i);
                        const bool improves = rs < ef || d < pdist(w.R[rs - 1]);
                        if (!improves) continue;
                        const uint64_t x = pack(d, nid);
                        bool cold = COLD && w.b_count != 0 && x > w.b_min;
                        if (!cold) {
                            if (!make_room<COLD>(w, head, tail, 1, rs, ef)) return -1;
                            cold = COLD && w.b_count != 0 && x > w.b_min;
                        }
                        if (COLD && cold) {
                            if (!cold_append(w, 1u, x)) return -1;
                        } else {
#ifdef HNSW_DEVICE_CHECKS
                            if (!HNSW_CHK(w.chk, tail < w.cand_cap + 1, 5, tail)) return -1;
#endif
                            sorted_insert(w.C, head, tail, x);
                            ++tail;
                        }
                        if ((A >> i) & 1u) {
                            sorted_insert(w.R, 0, rs, x);
                            ++rs;
                            if (rs > ef) rs = ef;
                        }
                    }
                }
            }
            if (V != kFull) break;
        }
    }
    return int(rs);
}

// layer0 for a query that admits every node (no filter, no tombstones).
// Results and live candidates then share one ascending array U: every entry
// is a result, with an "expanded" bit below the id (upack), and the next
// expansion is the first unexpanded entry. A result evicted before it was
// expanded stays a candidate of the reference's unbounded heap only if its
// distance equals the new worst result's (any larger one would meet the stop
// rule first, search.rs:113-119), so those wait in the tie list T. The
// expansion order, the visited set and every comparison are those of
// layer0, so the results are the same; one merge per round instead of two.
// U lives in the candidate array's space (cand_cap + 1 >= ef_cap + 33), T in
// the results array's; the results are copied back to w.R at the end.
// Returns rs, or -1 when the query outgrows the scratch (retried).
template <int DK>
__device__ __forceinline__ int layer0_single(QueryCtx& c, uint64_t ep, uint32_t ef) {
    const DeviceIndexView& ix = c.a->ix;
    Ws& w = *c.w;
    const int lane = lane_id();
    uint64_t* U = w.C;
    uint64_t* T = w.R;
    if (w.bitmap_mode) {
        for (uint32_t i = lane; i < w.bitmap_words; i += 32) w.H[i] = 0;
    } else {
        clear_hash(w);
    }
    __syncwarp();
    const uint32_t hash_limit = (w.hash_cap >> 2) * 3;
    uint32_t visited = 1;
    if (lane == 0) {
        visit(w, pid(ep));
        U[0] = to_upack(ep);
    }
    __syncwarp();
    uint32_t rs = 1, nt = 0, nx = 0, lost = 0;
    for (;;) {
        // p: the next expansion; pn: the one after it, unless this round
        // inserts something before it (its list is prefetched into L2).
        uint32_t p = rs, pn = rs;
        for (uint32_t b = nx; b < rs; b += 32) {
            const uint32_t i = b + lane;
            const uint32_t M = __ballot_sync(kFull, i < rs && !(U[i] & 1ull));
            if (M) {
                p = b + uint32_t(__ffs(int(M)) - 1);
                const uint32_t M2 = M & (M - 1);
                if (M2) pn = b + uint32_t(__ffs(int(M2)) - 1);
                break;
            }
        }
        uint64_t cur;
        if (p < rs) {
            cur = U[p];
            __syncwarp();
            if (lane == 0) {
                U[p] = cur | 1ull;
                if (pn < rs) prefetch_l2(ix.adj0 + size_t(uint32_t(U[pn]) >> 1) * ix.m0p, ix.m0p * 4);
            }
            nx = p + 1;
        } else {
            if (nt == 0) break;
            cur = T[0];
            for (uint32_t b = 0; b + 1 < nt; b += 32) {
                const uint32_t i = b + lane;
                const uint64_t v = i + 1 < nt ? T[i + 1] : 0;
                __syncwarp();
                if (i + 1 < nt) T[i] = v;
            }
            --nt;
            nx = rs;
            if (rs >= ef && pdist(cur) > pdist(U[rs - 1])) break;
        }
        __syncwarp();
        c.cnt.exp0++;
#ifdef HNSW_DEVICE_CHECKS
        if (!HNSW_CHK(w.chk, (uint32_t(cur) >> 1) < ix.n, 3, uint32_t(cur) >> 1)) return -1;
#endif
        const uint32_t* row = ix.adj0 + size_t(uint32_t(cur) >> 1) * ix.m0p;
        for (uint32_t base = 0; base < ix.m0; base += 32) {
#ifdef HNSW_DEVICE_CHECKS
            uint32_t id = (base + lane < ix.m0) ? __ldg(row + base + lane) : kEmpty;
            if (!HNSW_CHK(w.chk, id == kEmpty || id < ix.n, 2, id)) id = kEmpty;
#else
            const uint32_t id = (base + lane < ix.m0) ? __ldg(row + base + lane) : kEmpty;
#endif
            const bool valid = id != kEmpty;
            const uint32_t V = __ballot_sync(kFull, valid);
            if (V == 0) break;
            if (!w.bitmap_mode && visited + __popc(V) > hash_limit) {
                if (!w.spill_bits) return -1;
                // Move the visited set into the warp's global bitmap.
                spill_visited(w);
            }
            bool retry = false;
            const bool fresh = visit_chunk(w, id, valid, &retry);
            if (retry) return -1;
            if (is_tc(DK)) {
                if (fresh) {
                    prefetch_l2(ix.tc_hi + size_t(id) * (ix.dt >> 3), ix.dt * 2);
                    if (DK == DK_TC3) prefetch_l2(ix.tc_lo + size_t(id) * (ix.dt >> 3), ix.dt * 2);
                }
            } else if (fresh && (DK != DK_ANY || !w.stage)) {
                if (DK == DK_ANY && c.quant) prefetch_l2(ix.codes + size_t(id) * ix.dc, ix.dc);
                else prefetch_l2(ix.vec + size_t(id) * ix.dp, ix.dp * 4);
            }
            const uint32_t F = __ballot_sync(kFull, fresh);
            visited += __popc(F);
            if (F != 0) {
                chunk_distances<DK>(c, id, F);
                c.cnt.dist0 += __popc(F);
                const float my_d = fresh ? w.fd[lane] : 0.0f;
                uint32_t P = F;
                if (rs >= ef) P &= __ballot_sync(kFull, fresh && my_d < pdist(U[rs - 1]));
                if (P == 0) {
                    if (V != kFull) break;
                    continue;
                }
                const bool inP = (P >> lane) & 1u;
                const uint64_t my_x = upack(my_d, id);
                const float dz = __fadd_rn(my_d, 0.0f);
                const unsigned same =
                    __match_any_sync(kFull, inP ? __float_as_uint(dz) : (0x7FC00000u | uint32_t(lane)));
                uint32_t pr = 0;
                bool tie = inP && __popc(same) > 1;
                if (inP) {
                    pr = lower_bound(U, 0, rs, my_x);
                    if (pr < rs && pdist(U[pr]) == my_d) tie = true;
                    if (pr > 0 && pdist(U[pr - 1]) == my_d) tie = true;
                }
                if (!__any_sync(kFull, tie)) {
                    // before: entries of P earlier in the list and below this
                    // one (the sequential admission test); below: all entries
                    // of P below this one (its rank among them).
                    uint32_t before = 0, below = 0;
                    for (uint32_t bits = P; bits; bits &= bits - 1) {
                        const int j = __ffs(bits) - 1;
                        const uint64_t xj = __shfl_sync(kFull, my_x, j);
                        const bool lt = xj < my_x;
                        below += lt ? 1u : 0u;
                        before += (lt && j < lane) ? 1u : 0u;
                    }
                    const uint32_t I = __ballot_sync(kFull, inP && pr + before < ef);
                    if (I) {
#ifdef HNSW_DEVICE_CHECKS
                        if (!HNSW_CHK(w.chk, rs + uint32_t(__popc(I)) <= w.cand_cap + 1, 6, rs)) return -1;
#endif
                        // Rank among I: the entries of P below, less those
                        // left out of I.
                        for (uint32_t bits = P & ~I; bits; bits &= bits - 1) {
                            const int j = __ffs(bits) - 1;
                            below -= (__shfl_sync(kFull, my_x, j) < my_x) ? 1u : 0u;
                        }
                        // fr/fd (256 bytes, dead until the next chunk's
                        // distances) hold the merge's new entries.
                        nx = min(nx, merge_gather(U, rs, I, my_x, pr, below, reinterpret_cast<uint64_t*>(w.fr)));
                        const uint32_t total = rs + uint32_t(__popc(I));
                        if (total > ef) {
                            const float wd = pdist(U[ef - 1]);
                            const uint32_t i = ef + uint32_t(lane);
                            const uint64_t v = i < total ? U[i] : 0;
                            uint32_t E = __ballot_sync(kFull, i < total && !(v & 1ull) && pdist(v) == wd);
                            while (E) {
                                const int j = __ffs(int(E)) - 1;
                                E &= E - 1;
                                tie_add(T, nt, __shfl_sync(kFull, v, j), wd, lost);
                            }
                            rs = ef;
                        } else {
                            rs = total;
                        }
                    }
                } else {
                    while (P) {
                        const int i = __ffs(P) - 1;
                        P &= P - 1;
                        const float d = __shfl_sync(kFull, my_d, i);
                        const uint32_t nid = __shfl_sync(kFull, id, i);
                        const bool improves = rs < ef || d < pdist(U[rs - 1]);
                        if (!improves) continue;
                        const uint32_t pos = sorted_insert(U, 0, rs, upack(d, nid));
                        nx = min(nx, pos);
                        if (++rs > ef) {
                            rs = ef;
                            const uint64_t v = U[ef];
                            if (!(v & 1ull) && pdist(v) == pdist(U[ef - 1])) tie_add(T, nt, v, pdist(v), lost);
                        }
                    }
                }
                // A full tie list would drop a live candidate: retry with
                // the general queue instead.
                if (lost) return -1;
            }
            if (V != kFull) break;
        }
    }
    __syncwarp();
    for (uint32_t i = lane; i < rs; i += 32) w.R[i] = from_upack(U[i]);
    __syncwarp();
    return int(rs);
}

// Exact scan of the nodes a selective filter admits (the planner's route,
// advised by src/hnsw/mod.rs:421-425): every admitted live node gets its f32
// distance in the reference kernel order, and the best ef by (distance, id)
// stay in w.R; the caller sorts them by (distance, key). Returns the count.
static __device__ int exact_scan(QueryCtx& c, uint32_t ef) {
    const DeviceIndexView& ix = c.a->ix;
    Ws& w = *c.w;
    const int lane = lane_id();
    c.quant = false;             // exact rows, not codes
    uint8_t* stage = w.stage;    // staged gathers are sized for the request's rows
    w.stage = nullptr;
    uint32_t rs = 0;
    const uint64_t nb = min(c.fnbits, uint64_t(ix.n));
    const uint32_t nwords = uint32_t((nb + 63) / 64);
    for (uint32_t w0 = 0; w0 < nwords; w0 += 32) {
        const uint32_t wi = w0 + uint32_t(lane);
        uint64_t word = wi < nwords ? __ldg(c.fbits + wi) : 0ull;
        if (wi + 1 == nwords && (nb & 63)) word &= (1ull << (nb & 63)) - 1ull;
        while (__any_sync(kFull, word != 0)) {
            bool has = word != 0;
            uint32_t id = 0;
            if (has) {
                id = wi * 64u + uint32_t(__ffsll(static_cast<long long>(word)) - 1);
                word &= word - 1ull;
            }
            has = has && !(ix.has_dead && ((__ldg(ix.dead + (id >> 5)) >> (id & 31)) & 1u));
            const uint32_t F = __ballot_sync(kFull, has);
            if (F == 0) continue;
            chunk_distances(c, id, F);
            c.cnt.dist0 += __popc(F);
            const float my_d = has ? w.fd[lane] : 0.0f;
            const uint64_t my_x = pack(my_d, id);
            const uint64_t worst = rs >= ef ? w.R[rs - 1] : ~0ull;
            const uint32_t P = __ballot_sync(kFull, has && my_x < worst);
            if (P) {
                batch_merge(w.R, 0, rs, P, my_x, ef);
                rs = min(rs + uint32_t(__popc(P)), ef);
            }
        }
    }
    w.stage = stage;
    return int(rs);
}

// Prepares the query (vector::check + normalisation, src/vector.rs:22-45,
// 90-104; and the int8 code, src/quantization.rs:73-81) into the workspace.
// Returns a status.
static __device__ int32_t prepare(QueryCtx& c, const float* q) {
    const DeviceIndexView& ix = c.a->ix;
    Ws& w = *c.w;
    const int lane = lane_id();
    const uint32_t dim = ix.dim;
    bool bad = false;
    for (uint32_t i = lane; i < ix.dp; i += 32) {
        float x = i < dim ? q[i] : 0.0f;
        bad |= !isfinite(x);
        w.qf[i] = x;
    }
    bad = __any_sync(kFull, bad);
    __syncwarp();
    if (bad) return ST_NON_FINITE;
    double norm = 0.0;
    if (lane == 0)
        for (uint32_t i = 0; i < dim; ++i) {
            double x = double(w.qf[i]);
            norm = __dadd_rn(norm, __dmul_rn(x, x));
        }
    norm = __shfl_sync(kFull, norm, 0);
    if (norm > double(3.40282346638528859812e+38F) / 8.0) return ST_NON_FINITE;  // f32::MAX / 8
    if (c.metric == 2) {
        if (norm == 0.0) return ST_ZERO;
        const double inv = __ddiv_rn(1.0, __dsqrt_rn(norm));
        for (uint32_t i = lane; i < dim; i += 32) w.qf[i] = __double2float_rn(__dmul_rn(double(w.qf[i]), inv));
        __syncwarp();
    }
    if (c.quant) {
        const float inv = __fdiv_rn(1.0f, ix.scale);
        int sq = 0;
        for (uint32_t i = lane; i < ix.dc; i += 32) {
            int8_t code = i < dim ? sq_encode1(w.qf[i], __ldg(ix.q_offset + i), inv) : int8_t(0);
            w.qc[i] = code;
            sq += int(code) * int(code);
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) sq += __shfl_xor_sync(kFull, sq, off);
        c.qnorm = sq;
        __syncwarp();
    }
    return ST_OK;
}

// One query, start to finish. Returns the status written. The inputs are
// row qi of the arguments (query, k, ef, filter), the outputs row qo.
// V: 0 lean, 1 cold-list variant, 2 single-array variant (every node admitted).
// DK: the distance kinds compiled in (DK_ANY unless V == 2).
template <int V, int DK = DK_ANY>
__device__ __forceinline__ int32_t run_query(const SearchArgs& a, Ws& w, uint32_t qi, uint32_t qo) {
    const DeviceIndexView& ix = a.ix;
    const int lane = lane_id();
    QueryCtx c;
    c.a = &a;
    c.w = &w;
    c.qi = qi;
    c.metric = ix.metric;
    // Codes exist only on quantized indexes; a quantized request on any
    // other index fails with QuantizationDisabled after validation.
    c.quant = DK == DK_ANY && a.quantized != 0 && ix.quantized != 0;
    c.s2 = __fmul_rn(ix.scale, ix.scale);
    c.qnorm = 0;
    c.use_filter = a.filter_bits != nullptr && (a.filter_used == nullptr || a.filter_used[qi] != 0);
    const size_t fsel = a.filter_ids ? size_t(a.filter_ids[qi]) : size_t(qi);
    c.fbits = a.filter_bits + (a.filter_stride ? fsel * a.filter_stride : 0);
    c.fnbits = a.filter_nbits;
    c.by_node = a.filter_by_node != 0;
    const uint32_t k = min(a.ks ? a.ks[qi] : a.k, a.out_stride);
    uint32_t ef = a.efs ? a.efs[qi] : a.ef;
    uint32_t count = 0;
    int32_t st = prepare(c, a.queries + size_t(qi) * ix.dim);
    if (st == ST_OK && a.quantized && !ix.quantized) st = ST_QDISABLED;
    if constexpr (is_tc(DK)) {
        if (st == ST_OK) tc_prepare_query<DK == DK_TC3>(c);
    }
    if (st == ST_OK && k != 0 && ix.live != 0 && ix.entry != kEmpty) {
        ef = max(ef, k);
        if (ef > w.ef_cap) return ST_OVERFLOW;
        int rs;
        if (a.planned && a.planned[qi]) {
            rs = exact_scan(c, ef);
        } else {
            // search_graph (src/hnsw/search.rs:146-161)
            float d0;
            if constexpr (is_tc(DK)) {
                chunk_distances<DK>(c, lane == 0 ? ix.entry : 0u, 1u);
                d0 = w.fd[0];
            } else {
                const int g8 = lane & 7;
                d0 = group_distance<DK>(c, ix.entry, g8);
            }
            c.cnt.dist_up++;
            uint64_t ep = pack(d0, ix.entry);
            for (uint32_t layer = ix.top; layer >= 1; --layer) ep = greedy_layer<DK>(c, ep, layer);
            if constexpr (V == 2) rs = layer0_single<DK>(c, ep, ef);
            else rs = layer0<V == 1, DK>(c, ep, ef);
            if (rs < 0) return ST_OVERFLOW;
        }
        // Quantized or tensor-core traversal: exact distances for the
        // survivors (src/hnsw/mod.rs:494-498).
        if (c.quant || is_tc(DK)) {
            const int g = lane >> 3, g8 = lane & 7;
            for (int r = 0; r < rs; r += 4) {
                int slot = r + g;
                uint32_t id = pid(w.R[slot < rs ? slot : 0]);
                float d = group_exact(c, id, g8);
                __syncwarp();
                if (slot < rs && g8 == 0) w.C[slot] = pack(d, id);
                __syncwarp();
            }
            for (int i = lane; i < rs; i += 32) w.R[i] = w.C[i];
            __syncwarp();
        }
        // Sort by (total_cmp distance, key) and keep k (src/hnsw/mod.rs:501-510).
        uint64_t* key_of = w.C;
        for (int i = lane; i < rs; i += 32) key_of[i] = ix.keys_are_ids ? uint64_t(pid(w.R[i])) : __ldg(ix.keys + pid(w.R[i]));
        __syncwarp();
        count = min(uint32_t(rs), k);
        for (int i = lane; i < rs; i += 32) {
            const uint32_t dk = uint32_t(w.R[i] >> 32);
            const uint64_t key = key_of[i];
            uint32_t rank = 0;
            for (int j = 0; j < rs; ++j) {
                const uint32_t ok = uint32_t(w.R[j] >> 32);
                const uint64_t okey = key_of[j];
                rank += (ok < dk || (ok == dk && okey < key)) ? 1u : 0u;
            }
            if (rank < k) {
                const size_t o = size_t(qo) * a.out_stride + rank;
                a.out_keys[o] = key;
                a.out_dist[o] = kdec(dk);
            }
        }
        __syncwarp();
    }
    if (a.publish) {
        __threadfence_system();
        __syncwarp();
    }
    if (lane == 0) {
#ifdef HNSW_DEVICE_CHECKS
        if (!HNSW_CHK(w.chk, qo < a.nq, 9, qo)) return st;
#endif
        a.out_count[qo] = st == ST_OK ? count : 0u;
        if (a.publish) __threadfence_system();
        a.out_status[qo] = st;
        if (a.counters) {
            a.counters[4 * size_t(qo) + 0] = c.cnt.dist0;
            a.counters[4 * size_t(qo) + 1] = c.cnt.exp0;
            a.counters[4 * size_t(qo) + 2] = c.cnt.dist_up;
            a.counters[4 * size_t(qo) + 3] = c.cnt.exp_up;
        }
    }
    return st;
}

__host__ __device__ __forceinline__ size_t align_up(size_t x, size_t a) { return (x + a - 1) & ~(a - 1); }

// The retry kernel keeps its heaps in shared memory up to this ef capacity
// (results + candidates: about 25 KB per warp at 1024).
__host__ __device__ __forceinline__ bool retry_shared_heaps(uint32_t ef_cap) { return ef_cap <= 1024; }

__host__ __device__ __forceinline__ size_t retry_bytes_per_warp(uint32_t dp, uint32_t dc, uint32_t ef_cap,
                                                                uint32_t tcb = 0) {
    size_t b = align_up(size_t(dp) * 4, 16) + align_up(size_t(dc), 16) + 256 + align_up(size_t(tcb), 16);
    if (retry_shared_heaps(ef_cap))
        b += align_up(size_t(ef_cap + 1) * 8, 16) + align_up(size_t(2 * ef_cap + 32 + 1) * 8, 16);
    return b;
}

static __device__ void carve(Ws& w, char* base, const DeviceIndexView& ix, const SearchGeometry& g) {
    const uint32_t ef_cap = g.ef_cap, cand_cap = g.cand_cap, hash_cap = g.hash_cap;
    size_t off = 0;
    w.qf = reinterpret_cast<float*>(base + off);
    off = align_up(off + size_t(ix.dp) * 4, 16);
    w.qc = reinterpret_cast<int8_t*>(base + off);
    off = align_up(off + size_t(ix.dc), 16);
    w.qt = reinterpret_cast<uint4*>(base + off);
    off = align_up(off + size_t(g.tc_bytes), 16);
    w.R = reinterpret_cast<uint64_t*>(base + off);
    off = align_up(off + size_t(ef_cap + 1) * 8, 16);
    w.C = reinterpret_cast<uint64_t*>(base + off);
    off = align_up(off + size_t(cand_cap + 1) * 8, 16);
    w.fr = reinterpret_cast<uint32_t*>(base + off);
    off += 32 * 4;
    w.fd = reinterpret_cast<float*>(base + off);
    off += 32 * 4;
    w.stage = nullptr;
    w.stage_rows = 0;
    w.stage_row_bytes = 0;
    w.fi = nullptr;
    w.fnorm = nullptr;
    if (g.stage_rows) {
        w.fi = reinterpret_cast<uint32_t*>(base + off);
        off += 32 * 4;
        w.fnorm = reinterpret_cast<int32_t*>(base + off);
        off += 32 * 4;
        w.stage = reinterpret_cast<uint8_t*>(base + off);
        w.stage_rows = g.stage_rows;
        w.stage_row_bytes = g.stage_row_bytes;
        off = align_up(off + size_t(g.stage_rows) * g.stage_row_bytes, 16);
    }
    w.H = reinterpret_cast<uint32_t*>(base + off);
    w.ef_cap = ef_cap;
    w.cand_cap = cand_cap;
    w.hash_cap = hash_cap;
    w.tag16 = g.tag16 != 0;
    w.tag_sh = g.tag_sh;
    w.tag_mask = g.tag_mask;
    w.bitmap_mode = false;
    w.bitmap_words = 0;
    w.spill_bits = nullptr;
    w.spill_words = 0;
    w.spill_cands = nullptr;
    w.spill_cand_cap = 0;
    w.H0 = w.H;
    w.C0 = w.C;
    w.cand_cap0 = cand_cap;
    w.spilled_bits = w.spilled_cands = false;
    w.pool = nullptr;
    w.pool_next = nullptr;
    w.pool_chunks = 0;
    w.tab = nullptr;
    w.tab_cap = 0;
    w.b_chunks = 0;
#ifdef HNSW_DEVICE_CHECKS
    w.chk = nullptr;
#endif
    cold_reset(w);
}

// Gives the warp its cold-list row of the pool (`slot` < cold_slots).
static __device__ void attach_cold(Ws& w, const SearchArgs& a, uint32_t slot, uint32_t* next) {
    if (!a.cold_pool || slot >= a.cold_slots) return;
    w.pool = a.cold_pool;
    w.pool_next = next;
    w.pool_chunks = a.cold_chunks;
    w.tab = a.cold_tab + size_t(slot) * a.cold_tab_cap;
    w.tab_cap = a.cold_tab_cap;
    if (a.cold_private) w.b_chunks = w.tab_cap;
}

// Clears a spill bitmap and points the workspace back at shared memory.
static __device__ void end_spill(Ws& w) {
    const int lane = lane_id();
    if (w.spilled_bits) {
        uint4* b = reinterpret_cast<uint4*>(w.spill_bits);
        for (uint32_t i = lane; i < (w.spill_words >> 2); i += 32) b[i] = make_uint4(0, 0, 0, 0);
        __threadfence_block();
        __syncwarp();
        w.H = w.H0;
        w.bitmap_mode = false;
        w.bitmap_words = 0;
        w.spilled_bits = false;
    }
    if (w.spilled_cands) {
        w.C = w.C0;
        w.cand_cap = w.cand_cap0;
        w.spilled_cands = false;
    }
}

// The fast kernel. V = 0: candidate queues spill to a per-warp global array
// and, beyond it, to the retry pass; V = 1: the shared array's upper half
// moves to the cold list directly (persistent warps only); V = 2: the
// single-array layer 0. PERSIST: persistent warps drain the work counter;
// otherwise a warp runs its block's query once. Each mode is its own kernel
// with one inlined traversal (measured at 1M x 128, ef = 64: a kernel
// carrying both modes' copies ran persistent warps at 3.18 ms against
// 2.34 ms plain, and one copy inside the persistent loop cost plain warps
// 4 %). The bounds (256 threads, 2 blocks per SM: at most 128 registers)
// steer the register allocation: with the thread bound alone the plain
// kernels were built with 64 registers and spills (2.71 ms), without
// bounds with 72 (2.64 ms); with both they take 124-128 and run 2.26 ms.
template <int V, int DK = DK_ANY, bool PERSIST = false>
__global__ void __launch_bounds__(256, 2) search_kernel(SearchArgs a, SearchGeometry g) {
    extern __shared__ __align__(16) char smem[];
    const uint32_t warp = threadIdx.x >> 5;
    Ws w;
    carve(w, smem + size_t(warp) * g.bytes_per_warp, a.ix, g);
#ifdef HNSW_DEVICE_CHECKS
    w.chk = a.chk;
#endif
    const int lane = lane_id();
    if constexpr (PERSIST) {
        const uint32_t slot = blockIdx.x * (blockDim.x >> 5) + warp;
        if (a.spill_bits && slot < a.spill_slots) {
            w.spill_bits = a.spill_bits + size_t(slot) * a.spill_words;
            w.spill_words = a.spill_words;
            if (V == 0 && a.spill_cands) {
                w.spill_cands = a.spill_cands + size_t(slot) * (a.spill_cand_cap + 1);
                w.spill_cand_cap = a.spill_cand_cap;
            }
        }
        if (V == 1) attach_cold(w, a, slot, a.cold_next);
        for (;;) {
            uint32_t qi = 0;
            if (lane == 0) qi = atomicAdd(a.work_next, 1u);
            qi = __shfl_sync(kFull, qi, 0);
            if (qi >= a.nq) break;
            const int32_t st = run_query<V, DK>(a, w, qi, qi);
            end_spill(w);
            if (st == ST_OVERFLOW && lane == 0) {
                a.overflow_list[atomicAdd(a.overflow_count, 1u)] = qi;
                a.out_status[qi] = ST_OVERFLOW;
            }
        }
    } else {
        const uint32_t qi = blockIdx.x * (blockDim.x >> 5) + warp;
        if (qi >= a.nq) return;
        if (run_query<V, DK>(a, w, qi, qi) == ST_OVERFLOW && lane == 0) {
            a.overflow_list[atomicAdd(a.overflow_count, 1u)] = qi;
            a.out_status[qi] = ST_OVERFLOW;
        }
    }
}

// Retry pass: each warp owns a visited bitmap over all nodes and a cold
// candidate list; its results and candidate arrays sit in shared memory when
// ef fits (retry_shared_heaps) and in global memory otherwise. It takes
// overflowed queries in turn.
template <int DK = DK_ANY>
__global__ void __launch_bounds__(128) search_retry_kernel(SearchArgs a) {
    extern __shared__ __align__(16) char smem[];
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t gw = blockIdx.x * (blockDim.x >> 5) + warp;
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
    const DeviceIndexView& ix = a.ix;
    Ws w;
    // Query vectors and small buffers in shared memory, then the heaps when
    // they fit; the visited set in global memory.
    const bool sh = retry_shared_heaps(a.g_ef_cap);
    const uint32_t tcb = tc_query_bytes(a);
    const size_t per = retry_bytes_per_warp(ix.dp, ix.dc, a.g_ef_cap, tcb);
    char* base = smem + size_t(warp) * per;
    w.qf = reinterpret_cast<float*>(base);
    w.qc = reinterpret_cast<int8_t*>(base + align_up(size_t(ix.dp) * 4, 16));
    w.fr = reinterpret_cast<uint32_t*>(base + align_up(size_t(ix.dp) * 4, 16) + align_up(size_t(ix.dc), 16));
    w.fd = reinterpret_cast<float*>(w.fr + 32);
    w.qt = reinterpret_cast<uint4*>(base + align_up(size_t(ix.dp) * 4, 16) + align_up(size_t(ix.dc), 16) + 256);
    w.stage = nullptr;
    w.stage_rows = 0;
    w.stage_row_bytes = 0;
    w.fi = nullptr;
    w.fnorm = nullptr;
    if (sh) {
        char* heaps = base + align_up(size_t(ix.dp) * 4, 16) + align_up(size_t(ix.dc), 16) + 256 + align_up(size_t(tcb), 16);
        w.R = reinterpret_cast<uint64_t*>(heaps);
        w.C = reinterpret_cast<uint64_t*>(heaps + align_up(size_t(a.g_ef_cap + 1) * 8, 16));
        w.cand_cap = 2 * a.g_ef_cap + 32;
    } else {
        w.R = a.g_results + size_t(gw) * (a.g_ef_cap + 1);
        w.C = a.g_cands + size_t(gw) * (a.g_cand_cap + 1);
        w.cand_cap = a.g_cand_cap;
    }
    w.H = a.g_visited + size_t(gw) * a.g_visited_words;
    w.ef_cap = a.g_ef_cap;
    w.hash_cap = 0;
    w.tag16 = false;
    w.tag_sh = w.tag_mask = 0;
    w.bitmap_mode = true;
    w.bitmap_words = uint32_t(a.g_visited_words);
    w.spill_bits = nullptr;
    w.spill_words = 0;
    w.spill_cands = nullptr;
    w.spill_cand_cap = 0;
    w.H0 = w.H;
    w.C0 = w.C;
    w.cand_cap0 = w.cand_cap;
#ifdef HNSW_DEVICE_CHECKS
    w.chk = a.chk;
#endif
    w.spilled_bits = w.spilled_cands = false;
    w.pool = nullptr;
    w.pool_next = nullptr;
    w.pool_chunks = 0;
    w.tab = nullptr;
    w.tab_cap = 0;
    w.b_chunks = 0;
    cold_reset(w);
    attach_cold(w, a, gw, a.cold_next ? a.cold_next + 1 : nullptr);
    const uint32_t total = *a.overflow_count;
    for (uint32_t t = gw; t < total; t += nwarps) {
        const uint32_t qi = a.overflow_list[t];
#ifdef HNSW_DEVICE_CHECKS
        if (!HNSW_CHK(w.chk, qi < a.nq, 10, qi)) continue;
#endif
        // Writes ST_OVERFLOW again if even this scratch is too small; the
        // last-resort pass then takes the query.
        if (run_query<1, DK>(a, w, qi, qi) == ST_OVERFLOW && a.overflow_list2 && lane_id() == 0)
            a.overflow_list2[atomicAdd(a.overflow_count2, 1u)] = qi;
    }
}

}  // namespace dev
}  // namespace hnswgpu
