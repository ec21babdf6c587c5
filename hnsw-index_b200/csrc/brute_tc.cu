// Tensor-core brute-force scoring on sm_100a (tcgen05 + TMA + TMEM).
//
// Scores q . x for every (query, row) pair as one BF16 GEMM with FP32
// accumulation in tensor memory, either plainly (K = D, operands rounded to
// BF16) or with the 3-term split: operands [hi | lo] (each half padded to a
// multiple of 64 columns), and per K step three MMAs q_hi.x_hi, q_hi.x_lo,
// q_lo.x_hi on tiles loaded once, i.e. q.x up to the dropped q_lo.x_lo term. The epilogue turns each score
// into the metric's distance and either writes it densely (threshold sample)
// or keeps only (row, distance) pairs at or below a per-query threshold
// (candidate pass). Exact FP32 re-ranking of the survivors happens in
// brute_tc_rerank (K1 order), so the final results are those of
// BruteForceIndex::search_batch (src/brute.rs:169-180).
//
// Kernel structure (one CTA per SM, persistent over 128 x 256 output tiles):
//   warp 0      TMA producer: A (128 queries x 64 K) and B (256 rows x 64 K)
//               tiles into a shared-memory ring (128-byte swizzle): 4 stages
//               of one A and one B tile, or with the split 2 stages of
//               A_hi, A_lo, B_hi, B_lo (2/3 of the bytes per MMA);
//   warp 1      allocates 512 TMEM columns; one thread issues
//               tcgen05.mma (M=128, N=256, K=16) and tcgen05.commit;
//   warps 2..5  epilogue: tcgen05.ld of a 128 x 256 FP32 accumulator (two
//               accumulators alternate so the epilogue overlaps the next tile).
// Every mbarrier wait is bounded by a clock budget; on expiry the CTA sets an
// error word, drains, frees its TMEM and returns. No load is shared across a
// cluster.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>

#include "brute_tc.hpp"
#include "common.cuh"

namespace hnswgpu {
namespace tc {

constexpr uint32_t kTileM = 128, kTileN = 256, kTileK = 64;
constexpr uint32_t kABytes = kTileM * kTileK * 2;   // 16 KB
constexpr uint32_t kBBytes = kTileN * kTileK * 2;   // 32 KB
// Ring geometry per variant: tiles per stage of each operand, stages.
template <bool SPLIT3>
struct Ring {
    static constexpr int kTiles = SPLIT3 ? 2 : 1;
    static constexpr int kStages = SPLIT3 ? 2 : 4;
    static constexpr uint32_t kStageBytes = kTiles * (kABytes + kBBytes);  // 48 or 96 KB
};
constexpr uint32_t kTmemCols = 512;                   // two 256-column accumulators
constexpr int kThreads = 192;
constexpr long long kWaitBudget = 4000000000ll;       // drain waits, clock cycles (~2 s)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase with the given parity; false (and the error word set)
// if the clock budget runs out or another role already failed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t* err, long long budget) {
    const long long t0 = clock64();
    for (uint32_t i = 0;; ++i) {
        if (mbar_try(bar, parity)) return true;
        if ((i & 255) == 255) {
            if (*reinterpret_cast<volatile uint32_t*>(err)) return false;
            if (clock64() - t0 > budget) {
                atomicExch(err, 1u);
                return false;
            }
        }
    }
}

// Brings one box of the tensor map into L2 (no shared memory, no barrier).
__device__ __forceinline__ void tma_prefetch_l2(const CUtensorMap* map, int x, int y) {
    asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global [%0, {%1, %2}];" ::"l"(reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y)
                 : "memory");
}

// The base-row operand of a CTA's next tile, into L2 while the current tile
// runs: the CTAs of one round work on one or two n-tiles and reach each K
// chunk together, so without it every one of them waits on the same DRAM
// fetch. A CTA prefetches the chunks k = its index mod 4, 4 + that, ... of
// its next tile when the next tile's n-tile differs from the current one
// (the CTAs sharing that n-tile cover all chunks between them).
__device__ __forceinline__ void prefetch_next_b(const CUtensorMap* map, uint32_t nt, uint32_t nt_next, uint32_t k_chunks,
                                                int kT, uint32_t lo_col, int rows, int row_off, uint32_t who) {
    if (nt_next == nt) return;
    for (uint32_t k = who & 3u; k < k_chunks; k += 4)
        for (int tt = 0; tt < kT; ++tt)
            tma_prefetch_l2(map, int(k * kTileK + uint32_t(tt) * lo_col), int(nt_next) * rows + row_off);
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// UMMA shared-memory descriptor of a K-major tile with 128-byte swizzle:
// rows of 128 B, 8-row groups 1024 B apart (SBO), version 1, layout 2.
__device__ __forceinline__ uint64_t umma_desc(uint32_t smem_addr) {
    uint64_t d = 0;
    d |= uint64_t((smem_addr >> 4) & 0x3FFF);        // start address
    d |= uint64_t(1) << 16;                          // leading byte offset (unused with swizzle)
    d |= uint64_t(1024 >> 4) << 32;                  // stride byte offset
    d |= uint64_t(1) << 46;                          // descriptor version
    d |= uint64_t(2) << 61;                          // 128-byte swizzle
    return d;
}

// Instruction descriptor: BF16 x BF16 -> F32, both K-major, M=128, N=256.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((kTileN >> 3) << 17) | ((kTileM >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) asm volatile("" : "+r"(v[i]));
}
// tcgen05.ld without the wait: the registers are valid only after
// tmem_wait_regs on the same array.
__device__ __forceinline__ void tmem_ld32_async(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
}
// Waits for this thread's tcgen05.ld and re-defines v after the wait, so
// that no use of v is scheduled before it.
__device__ __forceinline__ void tmem_wait_regs(uint32_t (&v)[32]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) asm volatile("" : "+r"(v[i]));
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Metric distance of one accumulator value (approximate q.x).
__device__ __forceinline__ float tile_distance(const TcScoreArgs& a, float s, float qn, uint32_t row) {
    if (a.metric == 0) return qn + (row < a.n ? __ldg(a.xnorm2 + row) : 0.0f) - 2.0f * s;
    if (a.metric == 1) return -s;
    return 1.0f - s;
}

// The epilogue's per-row constants in registers (the scan loop then reads
// no kernel argument, which a store could otherwise force it to reload).
struct EpiConsts {
    int metric;
    uint32_t n;
    const float* xnorm2;
};
__device__ __forceinline__ float row_distance(const EpiConsts& e, float s, float qn, uint32_t row) {
    if (e.metric == 0) return qn + (row < e.n ? __ldg(e.xnorm2 + row) : 0.0f) - 2.0f * s;
    if (e.metric == 1) return -s;
    return 1.0f - s;
}

// Dense epilogue (threshold sample pass): this lane's query q against the
// 256 rows row_base .. row_base + 255 held in TMEM columns taddr .. taddr +
// 255 of its lane; every distance of the sample's row range is written,
// four at a time (+inf past the last row). All 32 lanes call.
__device__ __forceinline__ void epilogue_dense(const TcScoreArgs& a, uint32_t taddr, uint32_t q, uint32_t row_base) {
    const bool qvalid = q < a.nq;
    const float qn = (qvalid && a.qnorm2) ? a.qnorm2[q] : 0.0f;
    const EpiConsts e{a.metric, a.n, a.xnorm2};
    for (uint32_t c = 0; c < kTileN / 32; ++c) {
        uint32_t v[32];
        __syncwarp();
        tmem_ld32(taddr + c * 32, v);
        const uint32_t row0 = row_base + c * 32;
        // The sample range starts at a.row0 (a multiple of 256) and holds a.ld
        // (a multiple of 256) rows, so a chunk lies wholly inside or outside.
        if (!qvalid || row0 < a.row0 || row0 >= a.row0 + a.ld) continue;
        float4* out = reinterpret_cast<float4*>(a.dense + size_t(q) * a.ld + (row0 - a.row0));
#pragma unroll
        for (int j = 0; j < 32; j += 4) {
            float d[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const uint32_t row = row0 + uint32_t(j + i);
                d[i] = row < e.n ? row_distance(e, __uint_as_float(v[j + i]), qn, row) : __int_as_float(0x7f800000);
            }
            out[j / 4] = make_float4(d[0], d[1], d[2], d[3]);
        }
    }
}

// Candidate-mode staging: per epilogue warp and lane up to kStageDepth
// entries in shared memory, as the f32 distance and the row's column within
// the tile (entry i of lane l at [i * 32 + l], so consecutive lanes hit
// consecutive words). A chunk of 32 columns adds at most 32, so a warp
// appends its staged entries before a chunk whenever a lane holds more than
// kStageDepth - 32.
constexpr uint32_t kStageDepth = 48;
// One more row per lane takes the stores of entries that do not pass, so the
// scan has no branch per element.
constexpr uint32_t kStageBytesPerWarp = (kStageDepth + 1) * 32 * 5;  // 7.7 KB

// Appends this lane's n staged entries to its query's candidates (one
// reservation).
__device__ __forceinline__ void flush_stage(const TcScoreArgs& a, const float* sd, const uint8_t* sr, uint32_t q,
                                            uint32_t row_base, uint32_t n) {
    const int lane = threadIdx.x & 31;
    if (n == 0) return;
    uint32_t slot = atomicAdd(a.cand_count + q, n);
    uint64_t* out = a.cand + size_t(q) * a.cand_cap;
    for (uint32_t i = 0; i < n; ++i, ++slot)
        if (slot < a.cand_cap)
            out[slot] = (uint64_t(__float_as_uint(sd[i * 32 + lane])) << 32) | (row_base + sr[i * 32 + lane]);
}

// The 32 accumulator columns v (tile columns col0 .. col0 + 31) of this
// lane's query: entries at or below the threshold are staged. Straight-line
// code: every entry is stored, one that does not pass into the spare row
// kStageDepth, and only a passing one advances n. `lim` is the number of
// valid columns (0 for a padding query). METRIC as in tile_distance.
template <int METRIC>
__device__ __forceinline__ void stage_chunk_m(const EpiConsts& e, const uint32_t (&v)[32], uint32_t row_base,
                                              uint32_t col0, uint32_t lim, float thr, float qn, float* sd,
                                              uint8_t* sr, uint32_t& n) {
    const uint32_t lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
        const float s = __uint_as_float(v[j]);
        float dist;
        if (METRIC == 0) {
            const uint32_t row = row_base + col0 + uint32_t(j);
            dist = qn + (row < e.n ? __ldg(e.xnorm2 + row) : 0.0f) - 2.0f * s;
        } else if (METRIC == 1) {
            dist = -s;
        } else {
            dist = 1.0f - s;
        }
        const bool pass = uint32_t(j) < lim && dist <= thr;
        const uint32_t at = (pass ? n : kStageDepth) * 32 + lane;
        sd[at] = dist;
        sr[at] = uint8_t(col0 + uint32_t(j));
        n += pass ? 1u : 0u;
    }
}
__device__ __forceinline__ void stage_chunk(const EpiConsts& e, const uint32_t (&v)[32], uint32_t row_base,
                                            uint32_t col0, uint32_t lim, float thr, float qn, float* sd, uint8_t* sr,
                                            uint32_t& n) {
    if (e.metric == 0) stage_chunk_m<0>(e, v, row_base, col0, lim, thr, qn, sd, sr, n);
    else if (e.metric == 1) stage_chunk_m<1>(e, v, row_base, col0, lim, thr, qn, sd, sr, n);
    else stage_chunk_m<2>(e, v, row_base, col0, lim, thr, qn, sd, sr, n);
}

// Candidate mode, one pass: the accumulator's eight 32-column chunks are
// read with the next load in flight while the current chunk is scanned;
// `release` runs as soon as the last chunk is in registers (the MMA warp may
// then reuse the accumulator), and the staged entries are appended after.
template <typename Release>
__device__ __forceinline__ void epilogue_candidates(const TcScoreArgs& a, uint32_t taddr, uint32_t q,
                                                    uint32_t row_base, float thr, float qn, unsigned char* stage,
                                                    Release release) {
    const EpiConsts e{a.metric, a.n, a.xnorm2};
    float* sd = reinterpret_cast<float*>(stage);
    uint8_t* sr = stage + (kStageDepth + 1) * 32 * 4;
    // Valid columns of this tile for this lane's query.
    const uint32_t valid = q < a.nq ? (row_base < e.n ? min(e.n - row_base, kTileN) : 0u) : 0u;
    uint32_t n = 0;
    uint32_t va[32], vb[32];
    tmem_ld32_async(taddr, va);
    tmem_wait_regs(va);
#pragma unroll 1
    for (uint32_t c = 0; c < kTileN / 32; c += 2) {
        tmem_ld32_async(taddr + (c + 1) * 32, vb);
        if (__any_sync(0xFFFFFFFFu, n > kStageDepth - 32)) {
            flush_stage(a, sd, sr, q, row_base, n);
            n = 0;
        }
        __syncwarp();
        stage_chunk(e, va, row_base, c * 32, valid > c * 32 ? min(valid - c * 32, 32u) : 0u, thr, qn, sd, sr, n);
        __syncwarp();
        tmem_wait_regs(vb);
        if (c + 2 < kTileN / 32) tmem_ld32_async(taddr + (c + 2) * 32, va);
        else release();
        if (__any_sync(0xFFFFFFFFu, n > kStageDepth - 32)) {
            flush_stage(a, sd, sr, q, row_base, n);
            n = 0;
        }
        __syncwarp();
        stage_chunk(e, vb, row_base, (c + 1) * 32, valid > (c + 1) * 32 ? min(valid - (c + 1) * 32, 32u) : 0u, thr,
                    qn, sd, sr, n);
        __syncwarp();
        if (c + 2 < kTileN / 32) tmem_wait_regs(va);
    }
    flush_stage(a, sd, sr, q, row_base, n);
    __syncwarp();
}

template <bool SPLIT3>
__global__ void __launch_bounds__(kThreads, 1)
    score_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                 const __grid_constant__ TcScoreArgs a) {
    constexpr int kStages = Ring<SPLIT3>::kStages, kT = Ring<SPLIT3>::kTiles;
    constexpr uint32_t kStageBytes = Ring<SPLIT3>::kStageBytes;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte alignment for the swizzled tiles. Stage s holds kT A tiles
    // (hi, lo) then kT B tiles.
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    auto tileA = [&](uint32_t s, int t) { return smem + s * kStageBytes + uint32_t(t) * kABytes; };
    auto tileB = [&](uint32_t s, int t) { return smem + s * kStageBytes + kT * kABytes + uint32_t(t) * kBBytes; };
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
    uint64_t* empty = full + kStages;
    uint64_t* acc_full = empty + kStages;
    uint64_t* acc_empty = acc_full + 2;
    uint64_t* mma_done = acc_empty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);
    // Candidate staging of the four epilogue warps, after 256 bytes of barriers.
    unsigned char* stage_base = smem + kStages * kStageBytes + 256;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t q_tiles = a.q_tiles;
    const uint32_t n_tiles = a.n_tile_end - a.n_tile_begin;
    const uint32_t total = q_tiles * n_tiles;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 4);  // one arrival per epilogue warp
        }
        mbar_init(mma_done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            uint32_t it = 0;
            bool ok = true;
            for (uint32_t t = blockIdx.x; ok && t < total; t += gridDim.x) {
                const uint32_t nt = a.n_tile_begin + t / q_tiles, qt = t % q_tiles;
                if (t + gridDim.x < total)
                    prefetch_next_b(&tmB, nt, a.n_tile_begin + (t + gridDim.x) / q_tiles, a.k_chunks, kT, a.lo_col,
                                    int(kTileN), 0, blockIdx.x);
                for (uint32_t k = 0; k < a.k_chunks; ++k) {
                    const uint32_t s = it % kStages, ph = (it / kStages) & 1u;
                    if (!mbar_wait(&empty[s], ph ^ 1u, a.err, a.wait_budget)) {
                        ok = false;
                        break;
                    }
                    mbar_expect_tx(&full[s], kStageBytes);
#pragma unroll
                    for (int tt = 0; tt < kT; ++tt) {
                        const int x = int(k * kTileK + uint32_t(tt) * a.lo_col);
                        tma_load_2d(tileA(s, tt), &tmA, &full[s], x, int(qt * kTileM));
                        tma_load_2d(tileB(s, tt), &tmB, &full[s], x, int(nt * kTileN));
                    }
                    ++it;
                }
            }
            // Let the copies still in flight land before the CTA can exit
            // (bounded waits; on the normal path these phases are complete).
            const uint32_t inflight = it < uint32_t(kStages) ? it : uint32_t(kStages);
            for (uint32_t j = 0; j < inflight; ++j) {
                const uint32_t i2 = it - 1 - j;
                const long long t0 = clock64();
                while (!mbar_try(&full[i2 % kStages], (i2 / kStages) & 1u) && clock64() - t0 < kWaitBudget) {
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            uint32_t it = 0, tile_it = 0;
            // Test switch: nothing arrives on mma_done before the commit
            // below, so this wait runs out and the CTA takes the error path.
            const bool stalled = a.stall && !mbar_wait(mma_done, 0, a.err, a.wait_budget);
            for (uint32_t t = stalled ? total : blockIdx.x; t < total; t += gridDim.x, ++tile_it) {
                const uint32_t b = tile_it & 1u, use = tile_it >> 1;
                if (!mbar_wait(&acc_empty[b], (use & 1u) ^ 1u, a.err, a.wait_budget)) break;
                tc_fence_after();
                const uint32_t d = tmem_base + b * kTileN;
                bool ok = true;
                for (uint32_t k = 0; k < a.k_chunks; ++k, ++it) {
                    const uint32_t s = it % kStages, ph = (it / kStages) & 1u;
                    if (!mbar_wait(&full[s], ph, a.err, a.wait_budget)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint64_t ah = umma_desc(smem_u32(tileA(s, 0)));
                    const uint64_t bh = umma_desc(smem_u32(tileB(s, 0)));
                    if (SPLIT3) {
                        const uint64_t al = umma_desc(smem_u32(tileA(s, kT - 1)));
                        const uint64_t bl = umma_desc(smem_u32(tileB(s, kT - 1)));
#pragma unroll
                        for (uint32_t j = 0; j < kTileK / 16; ++j) {
                            umma_bf16(d, ah + 2 * j, bh + 2 * j, (k | j) != 0 ? 1u : 0u);
                            umma_bf16(d, ah + 2 * j, bl + 2 * j, 1u);
                            umma_bf16(d, al + 2 * j, bh + 2 * j, 1u);
                        }
                    } else {
#pragma unroll
                        for (uint32_t j = 0; j < kTileK / 16; ++j)
                            umma_bf16(d, ah + 2 * j, bh + 2 * j, (k | j) != 0 ? 1u : 0u);
                    }
                    umma_commit(&empty[s]);
                }
                if (!ok) break;
                umma_commit(&acc_full[b]);
            }
            // Every MMA this thread issued has completed before TMEM is freed.
            umma_commit(mma_done);
            const long long t0 = clock64();
            while (!mbar_try(mma_done, 0) && clock64() - t0 < kWaitBudget) {
            }
        }
    } else {
        // Epilogue: warp w reads TMEM lanes 32*(w%4) .. +31, i.e. those query rows.
        const uint32_t lane_base = 32u * uint32_t(warp & 3);
        unsigned char* stage = stage_base + size_t(warp - 2) * kStageBytesPerWarp;
        uint32_t tile_it = 0;
        for (uint32_t t = blockIdx.x; t < total; t += gridDim.x, ++tile_it) {
            const uint32_t nt = a.n_tile_begin + t / q_tiles, qt = t % q_tiles;
            const uint32_t b = tile_it & 1u, use = tile_it >> 1;
            const uint32_t q = qt * kTileM + lane_base + uint32_t(lane);
            // The query's threshold and norm load while the MMAs run.
            const float thr = (q < a.nq && a.thr) ? a.thr[q] : 0.0f;
            const float qn = (q < a.nq && a.qnorm2) ? a.qnorm2[q] : 0.0f;
            const bool got = __all_sync(0xFFFFFFFFu, mbar_wait(&acc_full[b], use & 1u, a.err, a.wait_budget));
            if (!got) break;
            tc_fence_after();
            const uint32_t taddr = tmem_base + (lane_base << 16) + b * kTileN;
            auto release = [&]() {
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&acc_empty[b]);
            };
            if (a.dense) {
                epilogue_dense(a, taddr, q, nt * kTileN);
                release();
            } else {
                epilogue_candidates(a, taddr, q, nt * kTileN, thr, qn, stage, release);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(kTmemCols));
    }
}

// ---------------------------------------------------------------------------
// Paired variant (cta_group::2): the two CTAs of a cluster compute one
// 256 x 256 output tile. CTA r holds queries r*128 .. r*128+127 of the pair's
// 256 (its A tile) and base rows r*128 .. r*128+127 of the tile's 256 (its
// half of B); one thread of CTA 0 issues tcgen05.mma with M = 256, which reads
// both CTAs' shared memory and writes each CTA's 128 query rows (x 256 rows)
// into its own tensor memory. Per CTA and K step that is half the B bytes of
// the single-CTA kernel for the same products, so more K steps fit in the
// ring (6 stages of 32 KB, or 3 of 64 KB with the split). Each CTA's TMA
// loads complete on its own barrier; CTA 1's warp 1 relays each completed
// stage to CTA 0 with a remote arrive. MMA completions are committed to both
// CTAs' barriers (one commit per CTA). Each CTA loads only its own tiles. Every
// wait is bounded as in score_kernel; the CTAs meet at a cluster barrier
// before tensor memory is freed, after CTA 0's MMAs and each CTA's copies
// have completed.
// ---------------------------------------------------------------------------
constexpr uint32_t kHalfN = kTileN / 2;                 // base rows per CTA
constexpr uint32_t kBHalfBytes = kHalfN * kTileK * 2;   // 16 KB
template <bool SPLIT3>
struct Ring2 {
    static constexpr int kTiles = SPLIT3 ? 2 : 1;
    static constexpr int kStages = SPLIT3 ? 3 : 6;
    static constexpr uint32_t kStageBytes = kTiles * (kABytes + kBHalfBytes);  // 32 or 64 KB
};
// Instruction descriptor: BF16 x BF16 -> F32, both K-major, M = 256 (pair), N = 256.
constexpr uint32_t kIdesc2 = (1u << 4) | (1u << 7) | (1u << 10) | ((kTileN >> 3) << 17) | ((256u >> 4) << 24);

__device__ __forceinline__ void umma_bf16_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(kIdesc2), "r"(accumulate));
}
// Arrives (once) on the barrier at `bar`'s offset in every CTA of `mask`
// when this thread's MMAs so far have completed: one commit per CTA, each to
// that CTA's barrier by its shared::cluster address (mapa).
__device__ __forceinline__ void umma_commit_pair(uint64_t* bar, uint16_t mask) {
    for (uint32_t r = 0; r < 2; ++r) {
        if (!((mask >> r) & 1u)) continue;
        uint32_t addr;
        asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(addr) : "r"(smem_u32(bar)), "r"(r));
        asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(addr)
                     : "memory");
    }
}
__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
// Arrive on the barrier at `bar`'s offset in CTA `rank` of the cluster.
__device__ __forceinline__ void mbar_arrive_remote(uint64_t* bar, uint32_t rank) {
    uint32_t remote;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(smem_u32(bar)), "r"(rank));
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(remote) : "memory");
}
// mbar_wait for a barrier that threads of the peer CTA arrive on (remote
// arrivals with release at cluster scope): the acquire is at cluster scope too.
__device__ __forceinline__ bool mbar_try_cluster(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* bar, uint32_t parity, uint32_t* err, long long budget) {
    const long long t0 = clock64();
    for (uint32_t i = 0;; ++i) {
        if (mbar_try_cluster(bar, parity)) return true;
        if ((i & 255) == 255) {
            if (*reinterpret_cast<volatile uint32_t*>(err)) return false;
            if (clock64() - t0 > budget) {
                atomicExch(err, 1u);
                return false;
            }
        }
    }
}
__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

template <bool SPLIT3>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreads, 1)
    score_pair_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                      const __grid_constant__ TcScoreArgs a) {
    constexpr int kStages = Ring2<SPLIT3>::kStages, kT = Ring2<SPLIT3>::kTiles;
    constexpr uint32_t kStageBytes = Ring2<SPLIT3>::kStageBytes;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // Both CTAs lay shared memory out identically: the MMA reads the peer's
    // operands at the same offsets.
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    auto tileA = [&](uint32_t s, int t) { return smem + s * kStageBytes + uint32_t(t) * kABytes; };
    auto tileB = [&](uint32_t s, int t) { return smem + s * kStageBytes + kT * kABytes + uint32_t(t) * kBHalfBytes; };
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
    uint64_t* peer_full = full + kStages;
    uint64_t* empty = peer_full + kStages;
    uint64_t* acc_full = empty + kStages;
    uint64_t* acc_empty = acc_full + 2;
    uint64_t* mma_done = acc_empty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);
    // Candidate staging of the four epilogue warps, after 256 bytes of barriers.
    unsigned char* stage_base = smem + kStages * kStageBytes + 256;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_rank();
    const bool leader = rank == 0;
    const uint32_t pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
    const uint32_t q_pairs = a.q_tiles >> 1;
    const uint32_t n_tiles = a.n_tile_end - a.n_tile_begin;
    const uint32_t total = q_pairs * n_tiles;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&peer_full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 8);  // four epilogue warps in each CTA
        }
        mbar_init(mma_done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // Producer (both CTAs): this CTA's A tile and half of B per K step.
            uint32_t it = 0;
            bool ok = true;
            for (uint32_t t = pair; ok && t < total; t += npairs) {
                const uint32_t nt = a.n_tile_begin + t / q_pairs, qp2 = t % q_pairs;
                if (t + npairs < total)
                    prefetch_next_b(&tmB, nt, a.n_tile_begin + (t + npairs) / q_pairs, a.k_chunks, kT, a.lo_col,
                                    int(kTileN), int(rank * kHalfN), pair);
                for (uint32_t k = 0; k < a.k_chunks; ++k) {
                    const uint32_t s = it % kStages, ph = (it / kStages) & 1u;
                    if (!mbar_wait(&empty[s], ph ^ 1u, a.err, a.wait_budget)) {
                        ok = false;
                        break;
                    }
                    mbar_expect_tx(&full[s], kStageBytes);
#pragma unroll
                    for (int tt = 0; tt < kT; ++tt) {
                        const int x = int(k * kTileK + uint32_t(tt) * a.lo_col);
                        tma_load_2d(tileA(s, tt), &tmA, &full[s], x, int((2 * qp2 + rank) * kTileM));
                        tma_load_2d(tileB(s, tt), &tmB, &full[s], x, int(nt * kTileN + rank * kHalfN));
                    }
                    ++it;
                }
            }
            const uint32_t inflight = it < uint32_t(kStages) ? it : uint32_t(kStages);
            for (uint32_t j = 0; j < inflight; ++j) {
                const uint32_t i2 = it - 1 - j;
                const long long t0 = clock64();
                while (!mbar_try(&full[i2 % kStages], (i2 / kStages) & 1u) && clock64() - t0 < kWaitBudget) {
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0 && !leader) {
            // Relay (CTA 1): each stage of this CTA that has landed is
            // reported to CTA 0's MMA issuer.
            uint32_t it = 0;
            bool ok = true;
            for (uint32_t t = pair; ok && t < total; t += npairs)
                for (uint32_t k = 0; k < a.k_chunks; ++k, ++it) {
                    const uint32_t s = it % kStages, ph = (it / kStages) & 1u;
                    if (!mbar_wait(&full[s], ph, a.err, a.wait_budget)) {
                        ok = false;
                        break;
                    }
                    mbar_arrive_remote(&peer_full[s], 0);
                }
        } else if (lane == 0) {
            // MMA issuer (CTA 0).
            uint32_t it = 0, tile_it = 0;
            for (uint32_t t = pair; t < total; t += npairs, ++tile_it) {
                const uint32_t b = tile_it & 1u, use = tile_it >> 1;
                if (!mbar_wait_cluster(&acc_empty[b], (use & 1u) ^ 1u, a.err, a.wait_budget)) break;
                tc_fence_after();
                const uint32_t d = tmem_base + b * kTileN;
                bool ok = true;
                for (uint32_t k = 0; k < a.k_chunks; ++k, ++it) {
                    const uint32_t s = it % kStages, ph = (it / kStages) & 1u;
                    if (!mbar_wait(&full[s], ph, a.err, a.wait_budget) ||
                        !mbar_wait_cluster(&peer_full[s], ph, a.err, a.wait_budget)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint64_t ah = umma_desc(smem_u32(tileA(s, 0)));
                    const uint64_t bh = umma_desc(smem_u32(tileB(s, 0)));
                    if (SPLIT3) {
                        const uint64_t al = umma_desc(smem_u32(tileA(s, kT - 1)));
                        const uint64_t bl = umma_desc(smem_u32(tileB(s, kT - 1)));
#pragma unroll
                        for (uint32_t j = 0; j < kTileK / 16; ++j) {
                            umma_bf16_pair(d, ah + 2 * j, bh + 2 * j, (k | j) != 0 ? 1u : 0u);
                            umma_bf16_pair(d, ah + 2 * j, bl + 2 * j, 1u);
                            umma_bf16_pair(d, al + 2 * j, bh + 2 * j, 1u);
                        }
                    } else {
#pragma unroll
                        for (uint32_t j = 0; j < kTileK / 16; ++j)
                            umma_bf16_pair(d, ah + 2 * j, bh + 2 * j, (k | j) != 0 ? 1u : 0u);
                    }
                    umma_commit_pair(&empty[s], 0x3);
                }
                if (!ok) break;
                umma_commit_pair(&acc_full[b], 0x3);
            }
            // Every MMA issued has completed before the CTAs part.
            umma_commit_pair(mma_done, 0x1);
            const long long t0 = clock64();
            while (!mbar_try(mma_done, 0) && clock64() - t0 < kWaitBudget) {
            }
        }
    } else {
        // Epilogue (both CTAs): this CTA's 128 query rows x the tile's 256 rows.
        const uint32_t lane_base = 32u * uint32_t(warp & 3);
        unsigned char* stage = stage_base + size_t(warp - 2) * kStageBytesPerWarp;
        uint32_t tile_it = 0;
        for (uint32_t t = pair; t < total; t += npairs, ++tile_it) {
            const uint32_t nt = a.n_tile_begin + t / q_pairs, qp2 = t % q_pairs;
            const uint32_t b = tile_it & 1u, use = tile_it >> 1;
            const uint32_t q = (2 * qp2 + rank) * kTileM + lane_base + uint32_t(lane);
            const float thr = (q < a.nq && a.thr) ? a.thr[q] : 0.0f;
            const float qn = (q < a.nq && a.qnorm2) ? a.qnorm2[q] : 0.0f;
            const bool got = __all_sync(0xFFFFFFFFu, mbar_wait(&acc_full[b], use & 1u, a.err, a.wait_budget));
            if (!got) break;
            tc_fence_after();
            const uint32_t taddr = tmem_base + (lane_base << 16) + b * kTileN;
            auto release = [&]() {
                tc_fence_before();
                __syncwarp();
                if (lane == 0) {
                    if (leader) mbar_arrive(&acc_empty[b]);
                    else mbar_arrive_remote(&acc_empty[b], 0);
                }
            };
            if (a.dense) {
                epilogue_dense(a, taddr, q, nt * kTileN);
                release();
            } else {
                epilogue_candidates(a, taddr, q, nt * kTileN, thr, qn, stage, release);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(kTmemCols));
    }
}

// Splits rows of fp32 values into BF16 operand rows: plain (kp columns: hi,
// zero padded) or 3-term (two halves of kp / 2 columns: hi, then lo = the
// BF16 rounding of x - hi, each zero padded). Rows >= n are zero.
__global__ void split_bf16_kernel(const float* __restrict__ src, uint32_t n, uint32_t dim, uint32_t src_stride,
                                  __nv_bfloat16* __restrict__ dst, uint32_t rows_padded, uint32_t kp, int terms) {
    const size_t total = size_t(rows_padded) * kp;
    const uint32_t half = terms == 3 ? kp / 2 : kp;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x) {
        const uint32_t r = uint32_t(i / kp), c = uint32_t(i % kp);
        const uint32_t seg = c / half, j = c % half;
        float out = 0.0f;
        if (r < n && j < dim) {
            const float x = src[size_t(r) * src_stride + j];
            const __nv_bfloat16 hi = __float2bfloat16_rn(x);
            out = seg == 0 ? __bfloat162float(hi) : __bfloat162float(__float2bfloat16_rn(x - __bfloat162float(hi)));
        }
        dst[i] = __float2bfloat16_rn(out);
    }
}

// Squared norms of fp32 rows (for the L2 epilogue).
__global__ void row_norms_kernel(const float* __restrict__ src, uint32_t n, uint32_t dim, uint32_t stride,
                                 float* __restrict__ out) {
    const uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= n) return;
    float s = 0.0f;
    for (uint32_t j = lane; j < dim; j += 32) {
        const float x = src[size_t(r) * stride + j];
        s = fmaf(x, x, s);
    }
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, off);
    if (lane == 0) out[r] = s;
}

// k-th smallest value of each query's row of `vals` (count entries, +inf
// padding allowed) by a 4-pass radix select on the order-preserving key; the
// threshold written is that value + margin[q] (or +inf when count < k).
__global__ void kth_threshold_kernel(const float* __restrict__ vals, uint32_t ld, const uint32_t* __restrict__ counts,
                                     const uint64_t* __restrict__ packed, uint32_t packed_cap, uint32_t nq, uint32_t k,
                                     const float* __restrict__ margin, float* __restrict__ thr_out) {
    __shared__ uint32_t hist[256];
    __shared__ uint32_t s_prefix, s_rank;
    const uint32_t q = blockIdx.x;
    if (q >= nq) return;
    const uint32_t n = counts ? min(counts[q], packed_cap) : ld;
    if (n < k || k == 0) {
        if (threadIdx.x == 0) thr_out[q] = __int_as_float(0x7f800000);
        return;
    }
    auto key_at = [&](uint32_t i) -> uint32_t {
        const float v = packed ? __uint_as_float(uint32_t(packed[size_t(q) * packed_cap + i] >> 32))
                               : vals[size_t(q) * ld + i];
        return dev::fkey(v);
    };
    uint32_t prefix = 0, rank = k;  // find the rank-th smallest key (1-based)
    for (int pass = 0; pass < 4; ++pass) {
        const int shift = 24 - 8 * pass;
        for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        const uint32_t mask_hi = pass == 0 ? 0u : (0xFFFFFFFFu << (32 - 8 * pass));
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint32_t key = key_at(i);
            if ((key & mask_hi) == (prefix & mask_hi)) atomicAdd(&hist[(key >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t acc = 0, digit = 0;
            for (; digit < 256; ++digit) {
                if (acc + hist[digit] >= rank) break;
                acc += hist[digit];
            }
            s_prefix = prefix | (digit << shift);
            s_rank = rank - acc;
        }
        __syncthreads();
        prefix = s_prefix;
        rank = s_rank;
        __syncthreads();
    }
    if (threadIdx.x == 0) thr_out[q] = dev::kdec(prefix) + margin[q];
}

// Per-query error margin 2E in distance units (see tc_margins).
__global__ void margins_kernel(const float* __restrict__ qnorm2, uint32_t nq, float max_xnorm, float eps, int metric,
                               uint32_t dim, float max_xnorm2, float* __restrict__ out) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const float qn2 = qnorm2[q];
    const float qn = sqrtf(qn2);
    float e = eps * qn * max_xnorm;  // bound on |approx dot - fp32 dot|
    if (metric == 0) e = 2.0f * e + float(dim + 4) * 5.96e-8f * (qn2 + max_xnorm2);
    out[q] = 2.0f * e * 1.0001f + 1e-30f;
}

}  // namespace tc

cudaError_t tc_margins(const float* qnorm2, uint32_t nq, float max_xnorm, float eps, int metric, uint32_t dim,
                       float* out, cudaStream_t stream) {
    if (nq == 0) return cudaSuccess;
    tc::margins_kernel<<<(nq + 255) / 256, 256, 0, stream>>>(qnorm2, nq, max_xnorm, eps, metric, dim,
                                                            max_xnorm * max_xnorm, out);
    return cudaGetLastError();
}

namespace {
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

bool make_map(CUtensorMap* map, const void* base, uint64_t rows, uint64_t kp, uint32_t box_rows) {
    auto fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {kp, rows};
    cuuint64_t strides[1] = {kp * 2};
    cuuint32_t box[2] = {tc::kTileK, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}
}  // namespace

uint32_t tc_k_padded(uint32_t dim, int terms) {
    const uint32_t half = (dim + tc::kTileK - 1) / tc::kTileK * tc::kTileK;
    return terms == 3 ? 2 * half : half;
}
uint32_t tc_rows_padded(uint32_t n, bool query_side, bool pairs) {
    const uint32_t t = query_side ? (pairs ? 2 * tc::kTileM : tc::kTileM) : tc::kTileN;
    return (std::max<uint32_t>(n, 1) + t - 1) / t * t;
}

cudaError_t tc_split(const float* src, uint32_t n, uint32_t dim, uint32_t src_stride, __nv_bfloat16* dst,
                     uint32_t rows_padded, uint32_t kp, int terms, bool query_side, cudaStream_t stream) {
    const size_t total = size_t(rows_padded) * kp;
    const uint32_t blocks = uint32_t(std::min<size_t>((total + 255) / 256, 148 * 64));
    (void)query_side;  // both operands use the same [hi | lo] layout
    tc::split_bf16_kernel<<<blocks, 256, 0, stream>>>(src, n, dim, src_stride, dst, rows_padded, kp, terms);
    return cudaGetLastError();
}

cudaError_t tc_row_norms(const float* src, uint32_t n, uint32_t dim, uint32_t stride, float* out, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    tc::row_norms_kernel<<<(n * 32 + 255) / 256, 256, 0, stream>>>(src, n, dim, stride, out);
    return cudaGetLastError();
}

cudaError_t tc_score(const __nv_bfloat16* A, uint32_t qp, const __nv_bfloat16* B, uint32_t np_, uint32_t kp,
                     const TcScoreArgs& args_in, int num_sms, cudaStream_t stream) {
    CUtensorMap ma, mb;
    const bool pairs = args_in.pairs != 0;
    if (pairs && qp % (2 * tc::kTileM) != 0) return cudaErrorInvalidValue;
    if (!make_map(&ma, A, qp, kp, tc::kTileM) || !make_map(&mb, B, np_, kp, pairs ? tc::kHalfN : tc::kTileN))
        return cudaErrorInvalidValue;
    TcScoreArgs a = args_in;
    a.q_tiles = qp / tc::kTileM;
    const bool split = a.terms == 3;
    a.lo_col = split ? kp / 2 : 0;
    a.k_chunks = (split ? kp / 2 : kp) / tc::kTileK;
    if (pairs) {
        const size_t smem2 = 1024 + size_t(split ? tc::Ring2<true>::kStages * tc::Ring2<true>::kStageBytes
                                                 : tc::Ring2<false>::kStages * tc::Ring2<false>::kStageBytes) +
                             256 + 4 * tc::kStageBytesPerWarp;
        auto kern2 = split ? tc::score_pair_kernel<true> : tc::score_pair_kernel<false>;
        cudaError_t e2 = raise_smem_limit(reinterpret_cast<const void*>(kern2));
        if (e2 != cudaSuccess) return e2;
        const uint32_t total2 = (a.q_tiles / 2) * (a.n_tile_end - a.n_tile_begin);
        if (total2 == 0) return cudaSuccess;
        const uint32_t npairs = std::max<uint32_t>(1, std::min<uint32_t>(total2, uint32_t(num_sms) / 2));
        kern2<<<2 * npairs, tc::kThreads, smem2, stream>>>(ma, mb, a);
        return cudaGetLastError();
    }
    const size_t smem = 1024 + size_t(split ? tc::Ring<true>::kStages * tc::Ring<true>::kStageBytes
                                            : tc::Ring<false>::kStages * tc::Ring<false>::kStageBytes) +
                        256 + 4 * tc::kStageBytesPerWarp;
    auto kern = split ? tc::score_kernel<true> : tc::score_kernel<false>;
    cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(kern));
    if (e != cudaSuccess) return e;
    const uint32_t total = a.q_tiles * (a.n_tile_end - a.n_tile_begin);
    if (total == 0) return cudaSuccess;
    const uint32_t grid = std::min<uint32_t>(total, uint32_t(num_sms));
    kern<<<grid, tc::kThreads, smem, stream>>>(ma, mb, a);
    return cudaGetLastError();
}

cudaError_t tc_kth_threshold(const float* vals, uint32_t ld, const uint32_t* counts, const uint64_t* packed,
                             uint32_t packed_cap, uint32_t nq, uint32_t k, const float* margin, float* thr_out,
                             cudaStream_t stream) {
    if (nq == 0) return cudaSuccess;
    tc::kth_threshold_kernel<<<nq, 256, 0, stream>>>(vals, ld, counts, packed, packed_cap, nq, k, margin, thr_out);
    return cudaGetLastError();
}

}  // namespace hnswgpu
