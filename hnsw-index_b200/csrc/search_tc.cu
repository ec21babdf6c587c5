// Tensor-core traversal kernels (hnsw_search_opts.traversal BF16 / BF16X3):
// the fast kernels of traverse.cuh and the retry pass built for the
// tensor-core distance kinds, in their own translation unit so that the f32
// kernels of search.cu are compiled exactly as without them; and the
// builder of the BF16 rows.
#include "traverse.cuh"

namespace hnswgpu {
namespace dev {

// One thread per 16-byte word of a node's tensor-core row: block b = c / 4
// of 32 dimensions, quad lane t = c % 4, its eight values in tc_row_pos
// order; the low parts are bf16(x - hi). Thread c == 0 also writes the f32
// squared norm (sequential sum) when `xnorm` is set.
__global__ void tc_rows_kernel(const float* __restrict__ vec, uint32_t n, uint32_t dim, uint32_t dp, uint32_t dt,
                               uint4* __restrict__ hi, uint4* __restrict__ lo, float* __restrict__ xnorm) {
    const uint32_t words = dt >> 3;
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= uint64_t(n) * words) return;
    const uint32_t node = uint32_t(i / words), c = uint32_t(i % words);
    const float* row = vec + size_t(node) * dp;
    const uint32_t b = c >> 2, t = c & 3u;
    __align__(16) __nv_bfloat16 h[8], l[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        // Inverse of tc_row_pos within the word.
        const uint32_t d = 32u * b + 16u * uint32_t(e >> 2) + 2u * t + 8u * uint32_t((e >> 1) & 1) + uint32_t(e & 1);
        const float x = d < dim ? row[d] : 0.0f;
        h[e] = __float2bfloat16_rn(x);
        l[e] = __float2bfloat16_rn(__fsub_rn(x, __bfloat162float(h[e])));
    }
    hi[i] = *reinterpret_cast<const uint4*>(h);
    if (lo) lo[i] = *reinterpret_cast<const uint4*>(l);
    if (xnorm && c == 0) {
        float s = 0.0f;
        for (uint32_t d = 0; d < dim; ++d) s = __fadd_rn(s, __fmul_rn(row[d], row[d]));
        xnorm[node] = s;
    }
}

}  // namespace dev

template <int DK>
static SearchKernel tc_kernel_for(int v, bool persistent) {
    using namespace dev;
    if (persistent) {
        if (v == 2) return search_kernel<2, DK, true>;
        return v == 1 ? search_kernel<1, DK, true> : search_kernel<0, DK, true>;
    }
    // Plain warps have no cold lists (V = 1 is persistent only).
    return v == 2 ? search_kernel<2, DK> : search_kernel<0, DK>;
}

SearchKernel tc_search_kernel(int v, int traversal, bool persistent) {
    return traversal == 2 ? tc_kernel_for<dev::DK_TC3>(v, persistent) : tc_kernel_for<dev::DK_TC1>(v, persistent);
}

RetryKernel tc_retry_kernel(int traversal) {
    return traversal == 2 ? dev::search_retry_kernel<dev::DK_TC3> : dev::search_retry_kernel<dev::DK_TC1>;
}

cudaError_t launch_tc_rows(const float* vec, uint32_t n, uint32_t dim, uint32_t dp, uint32_t dt, uint4* hi, uint4* lo,
                           float* xnorm, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    const uint64_t total = uint64_t(n) * (dt >> 3);
    const uint32_t threads = 256;
    dev::tc_rows_kernel<<<uint32_t((total + threads - 1) / threads), threads, 0, stream>>>(vec, n, dim, dp, dt, hi, lo,
                                                                                           xnorm);
    return cudaGetLastError();
}

}  // namespace hnswgpu
