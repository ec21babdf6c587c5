// Kernels and launchers of the query traversal whose device code is in
// traverse.cuh: the fast kernels for exact f32 and int8 traversal, the retry
// passes, the resident serving kernel, the selectivity planner and the int8
// encoder. The tensor-core traversal kernels are built in search_tc.cu.
#include "traverse.cuh"

namespace hnswgpu {
namespace dev {

// Resident serving kernel (ServeArgs, device.hpp). Global warp 0 is the
// doorbell: it copies the host's tail and stop words into device memory.
// The other warps claim published requests one at a time. A request with a
// filter, or on an index with tombstones, takes the cold-list variant;
// others take the single-array one (and the cold-list variant if they
// outgrow it). A query that outgrows even that publishes
// HNSW_ERR_SCRATCH_OVERFLOW and the host runs it again with the batch path's
// retry passes, after asking this kernel to leave (stop word) so that the
// retry kernels get SMs.
__global__ void __launch_bounds__(256) serve_kernel(SearchArgs a, SearchGeometry g, ServeArgs sv) {
    extern __shared__ __align__(16) char smem[];
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t gw = blockIdx.x * (blockDim.x >> 5) + warp;
    const int lane = lane_id();
    if (gw == 0) {
        // Doorbell. Polls the host words about once a microsecond; leaves
        // on stop, or once nothing new was published for twice the serving
        // warps' idle budget (they leave first).
        if (lane == 0) {
            uint64_t seen = *sv.tail;
            long long last = clock64();
            for (uint32_t it = 0; it < (1u << 30); ++it) {
                const uint32_t stop = *sv.host_stop;
                const uint64_t t = *sv.host_tail;
                if (t != seen) {
                    __threadfence_system();  // the ring rows behind the tail are visible before it
                    *sv.tail = t;
                    __threadfence();
                    seen = t;
                    last = clock64();
                }
                if (stop) {
                    *sv.stop = 1u;
                    __threadfence();
                    break;
                }
                if (clock64() - last > 2 * sv.idle_budget) break;
                __nanosleep(1000);
            }
        }
        return;
    }
    Ws w;
    carve(w, smem + size_t(warp) * g.bytes_per_warp, a.ix, g);
    if (a.spill_bits && gw < a.spill_slots) {
        w.spill_bits = a.spill_bits + size_t(gw) * a.spill_words;
        w.spill_words = a.spill_words;
    }
    attach_cold(w, a, gw, a.cold_next);
    const uint32_t dim = a.ix.dim;
    for (uint32_t served = 0; served < (1u << 30); ++served) {
        // Claim the next published request (lane 0), with a bounded wait.
        // The idle clock restarts whenever anything new is published, so the
        // warps leave together after a quiet period of the whole ring (not
        // one by one while requests still arrive for others to take).
        unsigned long long r = ~0ull;
        if (lane == 0) {
            long long idle0 = clock64();
            uint64_t seen_t = *sv.tail;
            uint32_t nap = 64;
            for (uint32_t it = 0; it < (1u << 30); ++it) {
                // The stop word first: a kernel asked to leave (server stop,
                // or to yield SMs to the retry passes) takes no new request;
                // published ones stay in the ring for the next launch.
                if (*sv.stop) break;
                const unsigned long long h = *reinterpret_cast<volatile unsigned long long*>(sv.claim);
                const uint64_t t = *sv.tail;
                if (h < t) {
                    if (atomicCAS(sv.claim, h, h + 1) == h) {
                        r = h;
                        break;
                    }
                    continue;  // another warp took it: look again at once
                }
                if (t != seen_t) {
                    seen_t = t;
                    idle0 = clock64();
                    nap = 64;
                }
                if (clock64() - idle0 > sv.idle_budget) break;
                __nanosleep(nap);
                nap = min(nap * 2u, 2048u);
            }
        }
        r = __shfl_sync(kFull, r, 0);
        if (r == ~0ull) break;
        __threadfence();  // the tail was read before the ring row
        const uint32_t slot = uint32_t(r % sv.ring_cap);
        // Copy the request into this warp's staging row (volatile loads: the
        // ring lives in mapped host memory and its rows are reused).
        for (uint32_t i = lane; i < dim; i += 32) sv.wq[size_t(gw) * dim + i] = sv.rq[size_t(slot) * dim + i];
        uint32_t bad = 0;
        if (lane == 0) {
            const int32_t fid = sv.rfid[slot];
            const uint32_t k = sv.rk[slot];
            if (r >= *sv.tail) bad = 1;
            else if (k == 0 || k > a.out_stride) bad = 2;
            else if (fid >= 0 && a.filter_bits != nullptr && uint32_t(fid) >= sv.filter_rows) bad = 3;
            sv.wk[gw] = k;
            sv.wef[gw] = sv.ref[slot];
            sv.wfu[gw] = fid >= 0 ? 1 : 0;
            sv.wfid[gw] = fid >= 0 ? uint32_t(fid) : 0u;
            if (bad && sv.err && atomicCAS(sv.err, 0u, bad) == 0u) sv.err[1] = uint32_t(r);
        }
        bad = __shfl_sync(kFull, bad, 0);
        __syncwarp();
        if (bad) {
            // Not run: the request is published with an argument error.
            if (lane == 0) {
                a.out_count[slot] = 0u;
                __threadfence_system();
                a.out_status[slot] = ST_BAD_ARGUMENT;
                if (sv.served) atomicAdd(sv.served, 1u);
            }
            __syncwarp();
            continue;
        }
        const bool general = a.ix.has_dead || (a.filter_bits != nullptr && sv.wfu[gw] != 0);
        int32_t st;
        if (general) {
            st = run_query<1>(a, w, gw, slot);
        } else {
            st = run_query<2>(a, w, gw, slot);
            if (st == ST_OVERFLOW) {
                // Outgrew the single array (a long run of equal distances):
                // the cold-list variant takes it on the same scratch.
                end_spill(w);
                st = run_query<1>(a, w, gw, slot);
            }
        }
        end_spill(w);
        if (st == ST_OVERFLOW) {
            __threadfence_system();
            __syncwarp();
            if (lane == 0) {
                a.out_count[slot] = 0u;
                __threadfence_system();
                a.out_status[slot] = ST_OVERFLOW;
            }
        }
        if (lane == 0 && sv.served) atomicAdd(sv.served, 1u);
        __syncwarp();
    }
}

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
    size_t b = al(size_t(dp) * 4) + al(dc) + al(size_t(g.ef_cap + 1) * 8) + al(size_t(g.cand_cap + 1) * 8) + 256 +
               size_t(g.hash_cap) * 4;
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
using SearchKernel = void (*)(SearchArgs, SearchGeometry);
static SearchKernel pick_search_kernel(const SearchArgs& args, const SearchGeometry& g) {
    if (!single_array_batch(args, g)) return g.cold ? dev::search_kernel<1> : dev::search_kernel<0>;
    if (args.quantized || g.stage_rows) return dev::search_kernel<2, dev::DK_ANY>;
    return args.ix.metric == 0 ? dev::search_kernel<2, dev::DK_L2> : dev::search_kernel<2, dev::DK_DOT>;
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
    for (SearchKernel kern : {g.cold ? dev::search_kernel<1> : dev::search_kernel<0>, dev::search_kernel<2, dev::DK_ANY>,
                              dev::search_kernel<2, dev::DK_L2>, dev::search_kernel<2, dev::DK_DOT>}) {
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
    const size_t smem = dev::retry_bytes_per_warp(args.ix.dp, args.ix.dc, args.g_ef_cap) * wpb;
    cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(dev::search_retry_kernel<dev::DK_ANY>));
    if (e != cudaSuccess) return e;
    dev::search_retry_kernel<dev::DK_ANY><<<(warps + wpb - 1) / wpb, 32 * wpb, smem, stream>>>(args);
    return cudaGetLastError();
}

cudaError_t launch_serve(const SearchArgs& args, const SearchGeometry& geo_in, const ServeArgs& sv, int num_sms,
                         cudaStream_t stream, uint32_t* warps_out) {
    SearchGeometry geo = geo_in;
    geo.bytes_per_warp = geometry_bytes_per_warp(geo, args.ix.dp, args.ix.dc);
    const size_t smem = size_t(geo.bytes_per_warp) * geo.warps_per_block;
    cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(dev::serve_kernel));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::serve_kernel, int(32 * geo.warps_per_block), smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    const uint32_t blocks = uint32_t(num_sms * per_sm);
    if (warps_out) *warps_out = blocks * geo.warps_per_block;
    dev::serve_kernel<<<blocks, 32 * geo.warps_per_block, smem, stream>>>(args, geo, sv);
    return cudaGetLastError();
}

cudaError_t serve_warps(const SearchGeometry& g_in, uint32_t dp, uint32_t dc, int num_sms, uint32_t* warps) {
    SearchGeometry g = g_in;
    g.bytes_per_warp = geometry_bytes_per_warp(g, dp, dc);
    const size_t smem = size_t(g.bytes_per_warp) * g.warps_per_block;
    cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(dev::serve_kernel));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::serve_kernel, int(32 * g.warps_per_block), smem);
    if (e != cudaSuccess) return e;
    *warps = uint32_t(std::max(per_sm, 1)) * g.warps_per_block * uint32_t(num_sms);
    return cudaSuccess;
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
