// Exact FP32 brute-force k-NN on CUDA cores, bit-identical to
// BruteForceIndex::search_filtered (src/brute.rs:131-160) with the AVX2
// kernels (src/kernels/x86.rs:32-131).
//
// Layout of the arithmetic: lane (c, l) = (lane >> 3, lane & 7) of a warp is
// AVX2 accumulator chain c, vector lane l. A warp scores a micro-tile of
// 4 queries x 8 rows: every lane runs the 32 FMA chains of its accumulator
// for the 32 (query, row) pairs, then a butterfly transpose-reduce adds the
// 32 accumulators of each pair in the reference order (bits 3, 4 of the lane
// = chains (c0+c1),(c2+c3) then their sum; bit 2 = v_l + v_{l+4}; bit 0 then
// bit 1 = the horizontal sum), leaving one pair's distance per lane.
// Each block keeps a per-query top-k (by total_cmp distance, then key) of its
// row slice; a merge kernel combines the slices.
#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "device.hpp"

namespace hnswgpu {
namespace dev {

constexpr int kQB = 16;      // queries per block (4 warps x 4)
constexpr int kRT = 8;       // rows per tile

// Orders (dk, row) entries by (distance key, key[row]).
__device__ __forceinline__ bool entry_less(uint64_t a, uint64_t b, const uint64_t* __restrict__ keys) {
    uint32_t da = uint32_t(a >> 32), db = uint32_t(b >> 32);
    if (da != db) return da < db;
    return __ldg(keys + uint32_t(a)) < __ldg(keys + uint32_t(b));
}

// Warp-cooperative insert of x into the ascending list L[0, n) (room for one more).
__device__ __forceinline__ void list_insert(uint64_t* L, uint32_t n, uint64_t x, const uint64_t* keys) {
    const int lane = threadIdx.x & 31;
    uint32_t pos = 0;
    for (uint32_t b = 0; b < n; b += 32) {
        uint32_t i = b + lane;
        bool lt = i < n && entry_less(L[i], x, keys);
        pos += __popc(__ballot_sync(kFull, lt));
    }
    if (n > pos)
        for (int c = int((n - pos - 1) >> 5); c >= 0; --c) {
            uint32_t i = pos + uint32_t(c) * 32 + lane;
            bool mv = i < n;
            uint64_t v = mv ? L[i] : 0;
            __syncwarp();
            if (mv) L[i + 1] = v;
            __syncwarp();
        }
    if (lane == 0) L[pos] = x;
    __syncwarp();
}

// vector::check + normalisation of each query (one warp per query).
__global__ void brute_prep_kernel(BruteArgs a) {
    const uint32_t q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (q >= a.nq) return;
    const float* src = a.queries + size_t(q) * a.dim;
    float* dst = a.qprep + size_t(q) * a.dp;
    bool bad = false;
    for (uint32_t i = lane; i < a.dp; i += 32) {
        float x = i < a.dim ? src[i] : 0.0f;
        bad |= !isfinite(x);
        dst[i] = x;
    }
    bad = __any_sync(kFull, bad);
    __syncwarp();
    int32_t st = 0;
    if (bad) st = 3;
    double norm = 0.0;
    if (!bad && lane == 0)
        for (uint32_t i = 0; i < a.dim; ++i) {
            double x = double(dst[i]);
            norm = __dadd_rn(norm, __dmul_rn(x, x));
        }
    norm = __shfl_sync(kFull, norm, 0);
    if (st == 0 && norm > double(3.40282346638528859812e+38F) / 8.0) st = 3;
    if (st == 0 && a.metric == 2) {
        if (norm == 0.0) st = 4;
        else {
            const double inv = __ddiv_rn(1.0, __dsqrt_rn(norm));
            for (uint32_t i = lane; i < a.dim; i += 32) dst[i] = __double2float_rn(__dmul_rn(double(dst[i]), inv));
        }
    }
    if (lane == 0) a.out_status[q] = st;
}

// Butterfly transpose-reduce of 32 values per lane over the lane bits in
// the order 3, 4, 2, 0, 1. Afterwards v[0] of lane L holds pair
// p(L) = (b3 << 4) | (b4 << 3) | (b2 << 2) | (b0 << 1) | b1 of the bits of L.
__device__ __forceinline__ float butterfly32(float (&v)[32], int lane) {
    const int order[5] = {3, 4, 2, 0, 1};
#pragma unroll
    for (int s = 0; s < 5; ++s) {
        const int half = 16 >> s;
        const bool hi = (lane >> order[s]) & 1;
#pragma unroll
        for (int j = 0; j < half; ++j) {
            float send = hi ? v[j] : v[j + half];
            float keep = hi ? v[j + half] : v[j];
            float recv = __shfl_xor_sync(kFull, send, 1 << order[s]);
            v[j] = __fadd_rn(keep, recv);
        }
    }
    return v[0];
}

__device__ __forceinline__ int pair_of_lane(int L) {
    return (((L >> 3) & 1) << 4) | (((L >> 4) & 1) << 3) | (((L >> 2) & 1) << 2) | ((L & 1) << 1) | ((L >> 1) & 1);
}

// Whether query q admits row r under the optional filter.
__device__ __forceinline__ bool brute_admits(const BruteArgs& a, uint32_t q, uint32_t r) {
    if (!a.filter_bits || (a.filter_used && !a.filter_used[q])) return true;
    const size_t sel = a.filter_ids ? size_t(a.filter_ids[q]) : size_t(q);
    const uint64_t* bits = a.filter_bits + (a.filter_stride ? sel * a.filter_stride : 0);
    const uint64_t bit = a.filter_by_row ? uint64_t(r) : __ldg(a.keys + r);
    return bit < a.filter_nbits && ((__ldg(bits + (bit >> 6)) >> (bit & 63)) & 1ull);
}

template <bool L2>
__global__ void __launch_bounds__(128) brute_score_kernel(BruteArgs a, uint32_t kk) {
    extern __shared__ __align__(16) char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t dp = a.dp;
    float* sq = reinterpret_cast<float*>(smem);                 // kQB * dp
    float* sr = sq + size_t(kQB) * dp;                           // kRT * dp
    uint64_t* lists = reinterpret_cast<uint64_t*>(sr + size_t(kRT) * dp);  // kQB * (kk + 1)
    const uint32_t q0 = blockIdx.x * kQB;
    const uint32_t slice = blockIdx.y, nslices = gridDim.y;
    const uint32_t rows_per = (a.n + nslices - 1) / nslices;
    const uint32_t r_begin = min(a.n, slice * rows_per), r_end = min(a.n, r_begin + rows_per);
    // Stage the block's prepared queries.
    for (uint32_t i = threadIdx.x; i < kQB * dp; i += blockDim.x) {
        uint32_t qq = i / dp, j = i % dp;
        sq[i] = (q0 + qq < a.nq) ? a.qprep[size_t(q0 + qq) * dp + j] : 0.0f;
    }
    // Per-query list sizes live in registers of the owning warp.
    uint32_t lsize[4] = {0, 0, 0, 0};
    __syncthreads();
    const uint32_t nfull = a.dim >> 5;
    const uint32_t rem8 = (a.dim & 31) >> 3;
    const uint32_t tail0 = (nfull << 5) + (rem8 << 3);
    const int p = pair_of_lane(lane);
    const int my_q = p >> 3, my_r = p & 7;  // pair p = 8 * query + row
    for (uint32_t t0 = r_begin; t0 < r_end; t0 += kRT) {
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < kRT * dp / 4; i += blockDim.x) {
            uint32_t rr = (i * 4) / dp, j = (i * 4) % dp;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (t0 + rr < r_end) v = ldg_f4(a.base + size_t(t0 + rr) * dp + j);
            *reinterpret_cast<float4*>(sr + rr * dp + j) = v;
        }
        __syncthreads();
        float acc[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) acc[i] = 0.0f;
        const float* qw = sq + size_t(warp * 4) * dp;
        for (uint32_t k = 0; k < nfull; ++k) {
            float qv[4], rv[8];
#pragma unroll
            for (int i = 0; i < 4; ++i) qv[i] = qw[size_t(i) * dp + 32 * k + lane];
#pragma unroll
            for (int i = 0; i < 8; ++i) rv[i] = sr[size_t(i) * dp + 32 * k + lane];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    if (L2) {
                        float d = __fsub_rn(qv[i], rv[j]);
                        acc[8 * i + j] = __fmaf_rn(d, d, acc[8 * i + j]);
                    } else {
                        acc[8 * i + j] = __fmaf_rn(qv[i], rv[j], acc[8 * i + j]);
                    }
                }
        }
        // 8-wide remainder blocks into chain 0 (lanes 0..7).
        if (lane < 8)
            for (uint32_t s = 0; s < rem8; ++s) {
                const uint32_t e = 32 * nfull + 8 * s + lane;
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        float x = qw[size_t(i) * dp + e], y = sr[size_t(j) * dp + e];
                        if (L2) {
                            float d = __fsub_rn(x, y);
                            acc[8 * i + j] = __fmaf_rn(d, d, acc[8 * i + j]);
                        } else {
                            acc[8 * i + j] = __fmaf_rn(x, y, acc[8 * i + j]);
                        }
                    }
            }
        float s = butterfly32(acc, lane);
        for (uint32_t e = tail0; e < a.dim; ++e) {
            float x = qw[size_t(my_q) * dp + e], y = sr[size_t(my_r) * dp + e];
            if (L2) {
                float d = __fsub_rn(x, y);
                s = __fadd_rn(s, __fmul_rn(d, d));
            } else {
                s = __fadd_rn(s, __fmul_rn(x, y));
            }
        }
        const float dist = metric_from_sum(a.metric, s);
        const uint32_t row = t0 + uint32_t(my_r);
        const uint32_t qg = q0 + uint32_t(warp * 4 + my_q);
        const bool valid = row < r_end && qg < a.nq && brute_admits(a, qg, row);
        const uint64_t cand = (uint64_t(fkey(dist)) << 32) | row;
        // Per-query top-k update (rare after warm-up).
#pragma unroll
        for (int qq = 0; qq < 4; ++qq) {
            uint64_t* L = lists + size_t(warp * 4 + qq) * (kk + 1);
            const uint32_t n = lsize[qq];
            bool want = valid && my_q == qq && (n < kk || entry_less(cand, L[n - 1], a.keys));
            uint32_t W = __ballot_sync(kFull, want);
            while (W) {
                const int src = __ffs(W) - 1;
                W &= W - 1;
                const uint64_t x = __shfl_sync(kFull, cand, src);
                uint32_t m = lsize[qq];
                if (m >= kk && !entry_less(x, L[m - 1], a.keys)) continue;
                list_insert(L, m, x, a.keys);
                lsize[qq] = min(m + 1, kk);
            }
        }
    }
    // Write this slice's partial lists.
    for (int qq = 0; qq < 4; ++qq) {
        const uint32_t qg = q0 + uint32_t(warp * 4 + qq);
        if (qg >= a.nq) continue;
        const uint64_t* L = lists + size_t(warp * 4 + qq) * (kk + 1);
        uint64_t* out = a.part + (size_t(qg) * nslices + slice) * kk;
        for (uint32_t i = lane; i < kk; i += 32) out[i] = i < lsize[qq] ? L[i] : ~0ull;
    }
}

// Merges the per-slice lists of each query (one warp per query): repeated
// minimum over the slice heads, ties broken by key.
__global__ void brute_merge_kernel(BruteArgs a, uint32_t kk, uint32_t nslices) {
    const uint32_t q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (q >= a.nq) return;
    if (a.out_status[q] != 0 || a.k == 0) {
        if (lane == 0) a.out_count[q] = 0;
        return;
    }
    const uint64_t* P = a.part + size_t(q) * nslices * kk;
    uint32_t head[2] = {0, 0};  // lanes own slices lane and lane + 32
    const uint32_t want = min(a.k, a.n);
    uint32_t got = 0;
    for (; got < want; ++got) {
        uint64_t best = ~0ull;
        int bs = -1;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            uint32_t s = uint32_t(lane) + 32u * h;
            if (s < nslices && head[h] < kk) {
                uint64_t v = P[size_t(s) * kk + head[h]];
                if (v != ~0ull && (bs < 0 || entry_less(v, best, a.keys))) {
                    best = v;
                    bs = int(s);
                }
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            uint64_t ob = __shfl_xor_sync(kFull, best, off);
            int os = __shfl_xor_sync(kFull, bs, off);
            bool take = os >= 0 && (bs < 0 || entry_less(ob, best, a.keys) ||
                                    (!entry_less(best, ob, a.keys) && os < bs));
            if (take) {
                best = ob;
                bs = os;
            }
        }
        if (bs < 0) break;
        if (uint32_t(bs) == uint32_t(lane)) head[0]++;
        if (uint32_t(bs) == uint32_t(lane) + 32) head[1]++;
        if (lane == 0) {
            a.out_keys[size_t(q) * a.k + got] = __ldg(a.keys + uint32_t(best));
            a.out_dist[size_t(q) * a.k + got] = kdec(uint32_t(best >> 32));
        }
    }
    if (lane == 0) a.out_count[q] = got;
}

// Exact re-rank of tensor-core candidates (one warp per query): every
// candidate whose approximate distance is <= thr2[q] gets its FP32 distance
// in the reference kernel order; a top-k list ordered by (total_cmp distance,
// key) keeps the best (src/brute.rs:131-160). A query whose candidate list
// overflowed gets status 25 and is re-run by the exact FP32 kernels.
__global__ void brute_rerank_kernel(BruteArgs a, const uint64_t* __restrict__ cand,
                                    const uint32_t* __restrict__ cand_count, uint32_t cand_cap,
                                    const float* __restrict__ thr2, uint32_t kk) {
    extern __shared__ __align__(16) char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t q = blockIdx.x * (blockDim.x >> 5) + uint32_t(warp);
    uint64_t* L = reinterpret_cast<uint64_t*>(smem) + size_t(warp) * (kk + 1);
    uint32_t* pos = reinterpret_cast<uint32_t*>(reinterpret_cast<uint64_t*>(smem) + size_t(blockDim.x >> 5) * (kk + 1)) +
                    warp * 32;
    if (q >= a.nq) return;
    if (a.out_status[q] != 0) {
        if (lane == 0) a.out_count[q] = 0;
        return;
    }
    const uint32_t total = cand_count[q];
    if (total > cand_cap) {
        if (lane == 0) a.out_status[q] = 25;
        return;
    }
    const float t2 = thr2[q];
    const float* qv = a.qprep + size_t(q) * a.dp;
    const uint64_t* C = cand + size_t(q) * cand_cap;
    const int g = lane >> 3, g8 = lane & 7;
    uint32_t size = 0;
    for (uint32_t base = 0; base < total; base += 32) {
        const uint32_t i = base + uint32_t(lane);
        uint32_t row = 0;
        bool pass = false;
        if (i < total) {
            const uint64_t c = C[i];
            pass = __uint_as_float(uint32_t(c >> 32)) <= t2;
            row = uint32_t(c);
        }
        const uint32_t P = __ballot_sync(kFull, pass);
        if (pass) pos[__popc(P & ((1u << lane) - 1u))] = row;
        __syncwarp();
        const uint32_t np = __popc(P);
        for (uint32_t r = 0; r < np; r += 4) {
            const uint32_t slot = r + uint32_t(g);
            const uint32_t rrow = pos[slot < np ? slot : 0];
            const float* xr = a.base + size_t(rrow) * a.dp;
            float sum = a.metric == 0 ? group_sum<true>(xr, qv, int(a.dim), g8) : group_sum<false>(xr, qv, int(a.dim), g8);
            const float d = metric_from_sum(a.metric, sum);
            const uint64_t e = (uint64_t(fkey(d)) << 32) | rrow;
            // Insert the (up to) four new entries one after another.
            for (int gg = 0; gg < 4; ++gg) {
                if (r + uint32_t(gg) >= np) break;
                const uint64_t x = __shfl_sync(kFull, e, gg * 8);
                if (size >= kk && !entry_less(x, L[size - 1], a.keys)) continue;
                list_insert(L, size, x, a.keys);
                size = min(size + 1, kk);
            }
        }
        __syncwarp();
    }
    const uint32_t want = min(a.k, a.n);
    for (uint32_t i = lane; i < size && i < want; i += 32) {
        a.out_keys[size_t(q) * a.k + i] = __ldg(a.keys + uint32_t(L[i]));
        a.out_dist[size_t(q) * a.k + i] = kdec(uint32_t(L[i] >> 32));
    }
    if (lane == 0) a.out_count[q] = min(size, want);
}

}  // namespace dev

cudaError_t launch_brute_prep(const BruteArgs& a, cudaStream_t stream) {
    dev::brute_prep_kernel<<<(a.nq * 32 + 127) / 128, 128, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_brute_rerank(const BruteArgs& a, const uint64_t* cand, const uint32_t* cand_count, uint32_t cand_cap,
                                const float* thr2, cudaStream_t stream) {
    const uint32_t kk = std::max<uint32_t>(1, std::min<uint32_t>(a.k, a.n ? a.n : 1));
    const uint32_t wpb = 4;
    const size_t smem = size_t(wpb) * (kk + 1) * 8 + size_t(wpb) * 32 * 4;
    cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(dev::brute_rerank_kernel));
    if (e != cudaSuccess) return e;
    dev::brute_rerank_kernel<<<(a.nq + wpb - 1) / wpb, 32 * wpb, smem, stream>>>(a, cand, cand_count, cand_cap, thr2, kk);
    return cudaGetLastError();
}

cudaError_t launch_brute_fp32(const BruteArgs& a, cudaStream_t stream) {
    const uint32_t kk = std::max<uint32_t>(1, std::min<uint32_t>(a.k, a.n ? a.n : 1));
    const uint32_t nslices = std::min<uint32_t>(a.tiles, 64);
    dev::brute_prep_kernel<<<(a.nq * 32 + 127) / 128, 128, 0, stream>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (a.n == 0 || a.k == 0) {
        BruteArgs b = a;
        dev::brute_merge_kernel<<<(a.nq * 32 + 127) / 128, 128, 0, stream>>>(b, kk, nslices);
        return cudaGetLastError();
    }
    const size_t smem = (size_t(dev::kQB) + dev::kRT) * a.dp * 4 + size_t(dev::kQB) * (kk + 1) * 8;
    dim3 grid((a.nq + dev::kQB - 1) / dev::kQB, nslices);
    if (a.metric == 0) {
        e = raise_smem_limit(reinterpret_cast<const void*>(dev::brute_score_kernel<true>));
        if (e != cudaSuccess) return e;
        dev::brute_score_kernel<true><<<grid, 128, smem, stream>>>(a, kk);
    } else {
        e = raise_smem_limit(reinterpret_cast<const void*>(dev::brute_score_kernel<false>));
        if (e != cudaSuccess) return e;
        dev::brute_score_kernel<false><<<grid, 128, smem, stream>>>(a, kk);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    dev::brute_merge_kernel<<<(a.nq * 32 + 127) / 128, 128, 0, stream>>>(a, kk, nslices);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Scratch for the allocation-free entry point
// (hnsw_gpu_brute_search_batch_noalloc). The prepared queries and the
// per-slice top-k lists live in this fixed array instead of memory the call
// allocates. Every GPU that loads the library holds it until the process
// exits. Host code must not pass the array's name to a kernel: on the host it
// is only a stand-in, so its device address is looked up once per device.
// ---------------------------------------------------------------------------
namespace {
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};
}  // namespace

cudaError_t noalloc_scratch_address(void** out) {
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[device] = p;
    }
    *out = g_noalloc_ptr[device];
    return cudaSuccess;
}

bool noalloc_layout(uint32_t nq, uint32_t dp, uint32_t kk, uint32_t want_slices, size_t* qprep_bytes,
                    uint32_t* slices) {
    const size_t q = (size_t(nq) * dp * 4 + 255) & ~size_t(255);
    if (q >= kNoAllocScratchBytes) return false;
    const size_t per_slice = size_t(nq) * kk * 8;
    const size_t fit = (kNoAllocScratchBytes - q) / per_slice;
    if (fit < 1) return false;
    *qprep_bytes = q;
    *slices = uint32_t(std::min<size_t>(fit, std::max<uint32_t>(1, want_slices)));
    return true;
}

}  // namespace hnswgpu
