// Kernels and launchers of the query traversal whose device code is in
// traverse.cuh: the fast kernels for exact f32 and int8 traversal, the retry
// passes, the selectivity planner and the int8 encoder. The tensor-core traversal kernels are built in search_tc.cu.
#include "traverse.cuh"

namespace hnswgpu {
namespace dev {

// One warp per query: whether its filter admits at most a.plan_max nodes.
__global__ void plan_kernel(SearchArgs a, uint8_t* planned) {
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    const DeviceIndexView& ix = a.ix;
    for (uint32_t qi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; qi < a.nq; qi += warps) {
        const bool use = a.filter_bits != nullptr && (a.filter_used == nullptr || a.filter_used[qi] != 0) &&
                         (ix.keys_are_ids || a.filter_by_node);
        bool plan = false;
        if (use) {
            const size_t fsel = a.filter_ids ? size_t(a.filter_ids[qi]) : size_t(qi);
            const uint64_t* bits = a.filter_bits + (a.filter_stride ? fsel * a.filter_stride : 0);
            const uint64_t nb = min(a.filter_nbits, uint64_t(ix.n));
            const uint32_t nwords = uint32_t((nb + 63) / 64);
            uint32_t count = 0;
            for (uint32_t w0 = 0; w0 < nwords && count <= a.plan_max; w0 += 32) {
                const uint32_t wi = w0 + uint32_t(lane);
                uint64_t word = wi < nwords ? __ldg(bits + wi) : 0ull;
                if (wi + 1 == nwords && (nb & 63)) word &= (1ull << (nb & 63)) - 1ull;
                count += __reduce_add_sync(kFull, uint32_t(__popcll(static_cast<long long>(word))));
            }
            plan = count <= a.plan_max;
        }
        if (lane == 0) planned[qi] = plan ? 1 : 0;
    }
}

__global__ void encode_codes_kernel(const float* __restrict__ vec, uint32_t n, uint32_t dim, uint32_t dp,
                                    uint32_t dc, const float* __restrict__ offset, float scale,
                                    int8_t* __restrict__ codes, int32_t* __restrict__ norms) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n) return;
    const float inv = __fdiv_rn(1.0f, scale);
    int sq = 0;
    for (uint32_t i = lane; i < dc; i += 32) {
        int8_t code = i < dim ? sq_encode1(vec[size_t(warp) * dp + i], offset[i], inv) : int8_t(0);
        codes[size_t(warp) * dc + i] = code;
        sq += int(code) * int(code);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) sq += __shfl_xor_sync(kFull, sq, off);
    if (lane == 0) norms[warp] = sq;
}

}  // namespace dev

uint32_t geometry_bytes_per_warp(const SearchGeometry& g, uint32_t dp, uint32_t dc) {
    auto al = [](size_t x) { return (x + 15) & ~size_t(15); };
    size_t b = al(size_t(dp) * 4) + al(dc) + al(g.tc_bytes) + al(size_t(g.ef_cap + 1) * 8) +
               al(size_t(g.cand_cap + 1) * 8) + 256 + size_t(g.hash_cap) * (g.tag16 ? 2 : 4);
    if (g.stage_rows) {
        const size_t rb = g.stage_row_bytes ? g.stage_row_bytes : size_t(dp) * 4;
        b += 256 + al(size_t(g.stage_rows) * rb);
    }
    return uint32_t(al(b));
}

// The single-array variant serves batches in which every query admits every
// node (no filter bitmaps, no tombstones) when the geometry leaves room for
// its arrays: ef_cap + 33 entries in the candidate array, the tie list in
// the results array.
static bool single_array_batch(const SearchArgs& args, const SearchGeometry& g) {
    return !args.filter_bits && !args.ix.has_dead && !args.planned && g.ef_cap >= dev::kTieCap &&
           g.cand_cap >= g.ef_cap + 32;
}

// The search kernel a batch takes: the single-array variant when it applies,
// built for its distance kind when the batch uses f32 rows loaded directly.
static SearchKernel pick_search_kernel(const SearchArgs& args, const SearchGeometry& g) {
    if (args.traversal) {
        const int v = single_array_batch(args, g) ? 2 : (g.cold ? 1 : 0);
        return tc_search_kernel(v, args.traversal, args.persistent != 0);
    }
    using namespace dev;
    if (args.persistent) {
        if (!single_array_batch(args, g)) return g.cold ? search_kernel<1, DK_ANY, true> : search_kernel<0, DK_ANY, true>;
        if (args.quantized || g.stage_rows) return search_kernel<2, DK_ANY, true>;
        return args.ix.metric == 0 ? search_kernel<2, DK_L2, true> : search_kernel<2, DK_DOT, true>;
    }
    // Cold lists need persistent warps' chunk tables: plain batches use V = 0.
    if (!single_array_batch(args, g)) return search_kernel<0>;
    if (args.quantized || g.stage_rows) return search_kernel<2, DK_ANY>;
    return args.ix.metric == 0 ? search_kernel<2, DK_L2> : search_kernel<2, DK_DOT>;
}

cudaError_t launch_search(const SearchArgs& args, const SearchGeometry& geo_in, int num_sms, cudaStream_t stream) {
    SearchGeometry geo = geo_in;
    geo.bytes_per_warp = geometry_bytes_per_warp(geo, args.ix.dp, args.ix.dc);
    const size_t smem = size_t(geo.bytes_per_warp) * geo.warps_per_block;
    const SearchKernel kern = pick_search_kernel(args, geo);
    cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(kern));
    if (e != cudaSuccess) return e;
    dim3 block(32 * geo.warps_per_block);
    dim3 grid;
    if (args.persistent) {
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, int(block.x), smem);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) per_sm = 1;
        grid = dim3(uint32_t(num_sms * per_sm));
        // Warps beyond the spill slots run without spill areas (overflow -> retry).
        (void)0;
    } else {
        grid = dim3((args.nq + geo.warps_per_block - 1) / geo.warps_per_block);
    }
    if (grid.x == 0) return cudaSuccess;
    kern<<<grid, block, smem, stream>>>(args, geo);
    return cudaGetLastError();
}

cudaError_t persistent_warps(const SearchGeometry& g_in, uint32_t dp, uint32_t dc, int num_sms, uint32_t* warps) {
    SearchGeometry g = g_in;
    g.bytes_per_warp = geometry_bytes_per_warp(g, dp, dc);
    const size_t smem = size_t(g.bytes_per_warp) * g.warps_per_block;
    // Spill slots for whichever variant a batch takes: the larger residency.
    int best = 1;
    using namespace dev;
    std::initializer_list<SearchKernel> kerns = {
        g.cold ? search_kernel<1, DK_ANY, true> : search_kernel<0, DK_ANY, true>, search_kernel<2, DK_ANY, true>,
        search_kernel<2, DK_L2, true>, search_kernel<2, DK_DOT, true>};
    // A geometry with tensor-core query operands is launched with those kernels.
    std::initializer_list<SearchKernel> tc_kerns = {tc_search_kernel(g.cold ? 1 : 0, 1, true),
                                                    tc_search_kernel(2, 1, true),
                                                    tc_search_kernel(g.cold ? 1 : 0, 2, true),
                                                    tc_search_kernel(2, 2, true)};
    for (SearchKernel kern : g.tc_bytes ? tc_kerns : kerns) {
        cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(kern));
        if (e != cudaSuccess) return e;
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, int(32 * g.warps_per_block), smem);
        if (e != cudaSuccess) return e;
        best = std::max(best, per_sm);
    }
    *warps = uint32_t(best) * g.warps_per_block * uint32_t(num_sms);
    return cudaSuccess;
}

cudaError_t launch_search_retry(const SearchArgs& args, uint32_t warps, cudaStream_t stream) {
    const uint32_t wpb = 4;
    const size_t smem =
        dev::retry_bytes_per_warp(args.ix.dp, args.ix.dc, args.g_ef_cap, tc_query_bytes(args)) * wpb;
    const RetryKernel kern = args.traversal ? tc_retry_kernel(args.traversal) : dev::search_retry_kernel<dev::DK_ANY>;
    cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(kern));
    if (e != cudaSuccess) return e;
    kern<<<(warps + wpb - 1) / wpb, 32 * wpb, smem, stream>>>(args);
    return cudaGetLastError();
}

cudaError_t launch_plan(const SearchArgs& args, uint8_t* planned, cudaStream_t stream) {
    if (args.nq == 0) return cudaSuccess;
    const uint32_t blocks = std::min<uint32_t>(148u * 8u, (args.nq * 32u + 255u) / 256u);
    dev::plan_kernel<<<blocks, 256, 0, stream>>>(args, planned);
    return cudaGetLastError();
}

cudaError_t launch_encode_codes(const float* vec, uint32_t n, uint32_t dim, uint32_t dp, uint32_t dc,
                                const float* offset, float scale, int8_t* codes, int32_t* norms, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    const uint32_t threads = 256;
    const uint64_t blocks = (uint64_t(n) * 32 + threads - 1) / threads;
    dev::encode_codes_kernel<<<uint32_t(blocks), threads, 0, stream>>>(vec, n, dim, dp, dc, offset, scale, codes, norms);
    return cudaGetLastError();
}

}  // namespace hnswgpu
