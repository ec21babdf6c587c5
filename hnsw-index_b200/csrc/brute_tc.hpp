// Tensor-core (tcgen05) scoring for the brute-force path.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace hnswgpu {

// Arguments of one scoring launch over row tiles [n_tile_begin, n_tile_end)
// (256 rows each) for all query tiles (128 queries each).
struct TcScoreArgs {
    uint32_t q_tiles = 0, k_chunks = 0;   // set by tc_score
    int terms = 1;                        // 1: plain BF16; 3: split (operands [hi | lo])
    uint32_t lo_col = 0;                  // set by tc_score: first column of the lo half
    uint32_t n_tile_begin = 0, n_tile_end = 0;
    uint32_t nq = 0, n = 0;               // valid queries / rows
    int metric = 0;
    const float* qnorm2 = nullptr;        // per query |q|^2 (L2)
    const float* xnorm2 = nullptr;        // per row |x|^2 (L2)
    // Dense mode: distances of rows [row0, row0 + ld) into dense[q * ld + row - row0].
    float* dense = nullptr;
    uint32_t row0 = 0, ld = 0;
    // Candidate mode: rows whose distance <= thr[q] are appended as
    // (f32 bits << 32 | row) to cand[q * cand_cap + slot], slot = cand_count[q]++.
    const float* thr = nullptr;
    uint32_t* cand_count = nullptr;
    uint64_t* cand = nullptr;
    uint32_t cand_cap = 0;
    uint32_t* err = nullptr;              // set to 1 if a bounded wait runs out
    // Clock budget of every pipeline wait (cycles); on expiry the CTA sets
    // *err, drains its copies and MMAs, frees its TMEM and returns.
    long long wait_budget = 4000000000ll;
    // Test switch for the timeout path: the MMA issuer first waits on a
    // barrier that nothing arrives at, so its bounded wait runs out.
    uint32_t stall = 0;
    // 1: the paired kernel (two CTAs of a cluster per 256 x 256 tile,
    // tcgen05.mma with cta_group::2); query tiles then come in pairs, so the
    // query operand rows must be padded to a multiple of 256.
    uint32_t pairs = 0;
};

uint32_t tc_k_padded(uint32_t dim, int terms);
uint32_t tc_rows_padded(uint32_t n, bool query_side, bool pairs = false);
// fp32 rows -> BF16 operand rows (terms 1: hi; terms 3: [hi | lo], halves of kp / 2).
cudaError_t tc_split(const float* src, uint32_t n, uint32_t dim, uint32_t src_stride, __nv_bfloat16* dst,
                     uint32_t rows_padded, uint32_t kp, int terms, bool query_side, cudaStream_t stream);
cudaError_t tc_row_norms(const float* src, uint32_t n, uint32_t dim, uint32_t stride, float* out, cudaStream_t stream);
cudaError_t tc_score(const __nv_bfloat16* A, uint32_t qp, const __nv_bfloat16* B, uint32_t np, uint32_t kp,
                     const TcScoreArgs& args, int num_sms, cudaStream_t stream);
// Per query: k-th smallest of a dense row (vals, ld) or of the packed
// candidates (packed, counts, cap), plus margin[q] -> thr_out[q] (+inf if
// fewer than k values).
cudaError_t tc_kth_threshold(const float* vals, uint32_t ld, const uint32_t* counts, const uint64_t* packed,
                             uint32_t packed_cap, uint32_t nq, uint32_t k, const float* margin, float* thr_out,
                             cudaStream_t stream);

// Margin 2E[q] with E = eps * |q| * max|x| (dot and cosine), or the L2
// equivalent (2E on the dot plus FP32 rounding of the norms).
cudaError_t tc_margins(const float* qnorm2, uint32_t nq, float max_xnorm, float eps, int metric, uint32_t dim,
                       float* out, cudaStream_t stream);

}  // namespace hnswgpu
