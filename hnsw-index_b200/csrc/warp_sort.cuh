// Warp-cooperative operations on ascending arrays of packed (distance key,
// id) entries, shared by the search and construction kernels.
#pragma once

#include "common.cuh"

namespace hnswgpu {
namespace dev {

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// Inserts x into the ascending array A[lo, hi) (capacity permitting one more
// entry). Returns the insertion position.
__device__ __forceinline__ uint32_t sorted_insert(uint64_t* A, uint32_t lo, uint32_t hi, uint64_t x) {
    const int lane = lane_id();
    uint32_t pos = lo;
    for (uint32_t base = lo; base < hi; base += 32) {
        uint32_t i = base + lane;
        bool lt = i < hi && A[i] < x;
        pos += __popc(__ballot_sync(kFull, lt));
    }
    // Shift [pos, hi) up by one, highest chunk first.
    if (hi > pos) {
        uint32_t n = hi - pos;
        for (int c = int((n - 1) >> 5); c >= 0; --c) {
            uint32_t i = pos + uint32_t(c) * 32 + lane;
            bool mv = i < hi;
            uint64_t v = mv ? A[i] : 0;
            __syncwarp();
            if (mv) A[i + 1] = v;
            __syncwarp();
        }
    }
    if (lane == 0) A[pos] = x;
    __syncwarp();
    return pos;
}

// First index in the ascending A[lo, hi) whose entry is not below x (one lane).
__device__ __forceinline__ uint32_t lower_bound(const uint64_t* A, uint32_t lo, uint32_t hi, uint64_t x) {
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (A[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Merges the entries x held by the lanes in S into the ascending A[lo, hi),
// keeping only positions below `limit` (truncation of the results array to
// ef). Entries are distinct. All lanes call.
__device__ __forceinline__ void batch_merge(uint64_t* A, uint32_t lo, uint32_t hi, uint32_t S, uint64_t x,
                                            uint32_t limit) {
    const int lane = lane_id();
    const bool in = (S >> lane) & 1u;
    uint32_t rank_s = 0;
    for (uint32_t bits = S; bits; bits &= bits - 1) {
        const int j = __ffs(bits) - 1;
        rank_s += (__shfl_sync(kFull, x, j) < x) ? 1u : 0u;
    }
    const uint32_t pa = in ? lower_bound(A, lo, hi, x) : hi;
    // The smallest new entry sits at the lowest insertion point.
    const uint32_t pmin = __reduce_min_sync(kFull, in ? pa : 0xFFFFFFFFu);
    if (hi > pmin) {
        for (int base = int((hi - 1) & ~31u); base >= int(pmin & ~31u); base -= 32) {
            const uint32_t k = uint32_t(base) + uint32_t(lane);
            const bool mv = k >= pmin && k < hi;
            const uint64_t v = mv ? A[k] : 0;
            uint32_t shift = 0;
            for (uint32_t bits = S; bits; bits &= bits - 1) {
                const int j = __ffs(bits) - 1;
                shift += (__shfl_sync(kFull, x, j) < v) ? 1u : 0u;
            }
            __syncwarp();
            if (mv && k + shift < limit) A[k + shift] = v;
            __syncwarp();
        }
    }
    if (in && pa + rank_s < limit) A[pa + rank_s] = x;
    __syncwarp();
}

__device__ __forceinline__ uint64_t warp_min_u64(uint64_t v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const uint64_t o = __shfl_xor_sync(kFull, v, off);
        v = o < v ? o : v;
    }
    return v;
}

__device__ __forceinline__ uint64_t warp_max_u64(uint64_t v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const uint64_t o = __shfl_xor_sync(kFull, v, off);
        v = o > v ? o : v;
    }
    return v;
}

// Layer-search entries: (fkey(d) << 32) | (id << 1) | expanded. The flag bit
// sits below the id, so the u64 order is still the (total_cmp distance, id)
// order of Candidate (src/hnsw/search.rs:36-44).
__device__ __forceinline__ uint64_t upack(float d, uint32_t id) { return (uint64_t(fkey(d)) << 32) | (uint64_t(id) << 1); }
__device__ __forceinline__ uint64_t to_upack(uint64_t x) { return (x & 0xFFFFFFFF00000000ull) | (uint64_t(uint32_t(x)) << 1); }
__device__ __forceinline__ uint64_t from_upack(uint64_t x) { return (x & 0xFFFFFFFF00000000ull) | (uint32_t(x) >> 1); }

// Merges the entries x of the lanes in S (distinct, none in A) into the
// ascending A[0, hi) (room for all of them). `at` is, in the lanes of S,
// lower_bound(A, 0, hi, x) when the caller has it already (else ~0u: it is
// computed here). Returns the lowest position written. All lanes call.
__device__ __forceinline__ uint32_t merge_all(uint64_t* A, uint32_t hi, uint32_t S, uint64_t x,
                                              uint32_t at = ~0u) {
    const int lane = lane_id();
    const bool in = (S >> lane) & 1u;
    uint32_t rank_s = 0;
    for (uint32_t bits = S; bits; bits &= bits - 1) {
        const int j = __ffs(bits) - 1;
        rank_s += (__shfl_sync(kFull, x, j) < x) ? 1u : 0u;
    }
    const uint32_t pa = in ? (at != ~0u ? at : lower_bound(A, 0, hi, x)) : hi;
    const uint32_t pmin = __reduce_min_sync(kFull, in ? pa : 0xFFFFFFFFu);
    if (hi > pmin) {
        for (int b = int((hi - 1) & ~31u); b >= int(pmin & ~31u); b -= 32) {
            const uint32_t k = uint32_t(b) + uint32_t(lane);
            const bool mv = k >= pmin && k < hi;
            const uint64_t v = mv ? A[k] : 0;
            uint32_t shift = 0;
            for (uint32_t bits = S; bits; bits &= bits - 1) {
                const int j = __ffs(bits) - 1;
                shift += (__shfl_sync(kFull, x, j) < v) ? 1u : 0u;
            }
            __syncwarp();
            if (mv) A[k + shift] = v;
            __syncwarp();
        }
    }
    if (in) A[pa + rank_s] = x;
    __syncwarp();
    return pmin;
}

// merge_all with the positions known: the lanes of S (distinct entries x,
// none in A) give their lower bound `pa` in the ascending A[0, hi) and their
// rank `rk` among S, so each new entry's final position is pa + rk. Every
// output position then gathers its entry instead of every old entry
// counting the new ones below it: per 32-position chunk one OR reduction
// collects the new entries' positions, an old entry at output o comes from
// A[o - (new entries at or below o)] and a new one from `scratch` (32
// entries, by rank). Chunks are rewritten from the top down and each is
// read before it is written; a source never lies above its output, so
// every source is read before its slot is overwritten. Room for hi + |S|
// entries. Returns the lowest position written. All lanes call.
__device__ __forceinline__ uint32_t merge_gather(uint64_t* A, uint32_t hi, uint32_t S, uint64_t x, uint32_t pa,
                                                 uint32_t rk, uint64_t* scratch) {
    const int lane = lane_id();
    const bool in = (S >> lane) & 1u;
    const uint32_t q = pa + rk;
    if (in) scratch[rk] = x;
    const uint32_t pmin = __reduce_min_sync(kFull, in ? pa : 0xFFFFFFFFu);
    const uint32_t total = hi + uint32_t(__popc(S));
    const uint32_t upto = (2u << lane) - 1u;  // lanes at or below this one
    __syncwarp();
    for (int c = int((total - 1) >> 5); c >= int(pmin >> 5); --c) {
        const uint32_t b = uint32_t(c) << 5;
        const uint32_t M = __reduce_or_sync(kFull, (in && q >= b && q < b + 32) ? 1u << (q - b) : 0u);
        const uint32_t nb = __reduce_add_sync(kFull, (in && q < b) ? 1u : 0u);
        const uint32_t o = b + uint32_t(lane);
        const uint32_t nle = nb + uint32_t(__popc(M & upto));
        const bool act = o >= pmin && o < total;
        uint64_t v = 0;
        if (act) v = ((M >> lane) & 1u) ? scratch[nle - 1] : A[o - nle];
        __syncwarp();
        if (act) A[o] = v;
        __syncwarp();
    }
    return pmin;
}

// batch_merge by gathering (as merge_gather): the lanes of S (distinct
// entries x, none in A[lo, hi)) merge into the ascending A[lo, hi), and
// positions at or above `limit` are dropped. `scratch` holds 32 entries.
// All lanes call.
__device__ __forceinline__ void batch_merge_gather(uint64_t* A, uint32_t lo, uint32_t hi, uint32_t S, uint64_t x,
                                                   uint32_t limit, uint64_t* scratch) {
    const int lane = lane_id();
    const bool in = (S >> lane) & 1u;
    uint32_t rk = 0;
    for (uint32_t bits = S; bits; bits &= bits - 1) {
        const int j = __ffs(bits) - 1;
        rk += (__shfl_sync(kFull, x, j) < x) ? 1u : 0u;
    }
    const uint32_t pa = in ? lower_bound(A, lo, hi, x) : hi;
    const uint32_t q = pa + rk;
    if (in) scratch[rk] = x;
    const uint32_t pmin = __reduce_min_sync(kFull, in ? pa : 0xFFFFFFFFu);
    const uint32_t end = min(hi + uint32_t(__popc(S)), limit);
    const uint32_t upto = (2u << lane) - 1u;
    __syncwarp();
    if (pmin < end) {
        for (int c = int((end - 1) >> 5); c >= int(pmin >> 5); --c) {
            const uint32_t b = uint32_t(c) << 5;
            const uint32_t M = __reduce_or_sync(kFull, (in && q >= b && q < b + 32) ? 1u << (q - b) : 0u);
            const uint32_t nb = __reduce_add_sync(kFull, (in && q < b) ? 1u : 0u);
            const uint32_t o = b + uint32_t(lane);
            const uint32_t nle = nb + uint32_t(__popc(M & upto));
            const bool act = o >= pmin && o < end;
            uint64_t v = 0;
            if (act) v = ((M >> lane) & 1u) ? scratch[nle - 1] : A[o - nle];
            __syncwarp();
            if (act) A[o] = v;
            __syncwarp();
        }
    }
}

constexpr uint32_t kTieCap = 32;

// A result evicted while unexpanded stays a candidate of the reference's
// unbounded queue; it can still be expanded only if its distance equals the
// worst result's (search.rs:113-119). Such entries (all of one distance)
// wait in the ascending tie list T; entries of a larger distance are dead.
__device__ __forceinline__ void tie_add(uint64_t* T, uint32_t& nt, uint64_t x, float wd, uint32_t& inexact) {
    if (nt && pdist(T[0]) > wd) nt = 0;
    if (nt >= kTieCap) {
        inexact = 1;
        return;
    }
    sorted_insert(T, 0, nt, x);
    ++nt;
}

}  // namespace dev
}  // namespace hnswgpu
