// Host side of the device graph construction: uploads a builder's graph,
// plans the waves, launches them back to back on one stream and writes the
// linked graph back into the builder.
//
// Wave plan. The first node of an empty graph becomes the entry point
// (link_parallel links it alone, src/hnsw/mod.rs:340-349). After that a wave
// links max(1, floor(linked * fraction)) nodes, at most max_wave, where
// `linked` counts the nodes already in the graph. A node whose level is above
// the current top level is linked alone and then becomes the entry point:
// the promotion lock of build.rs:52-66 serialises exactly those nodes. Levels
// are sampled from the node id (build.rs:19-28), so the plan, and with it the
// graph, depends only on the inputs and the two wave settings.
#include "gpu_build.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "build.hpp"
#include "capi_internal.hpp"

namespace hnswgpu {
namespace {

struct Wave {
    uint32_t first, count, entry, top, records;
};

struct DevMem {
    std::vector<void*> ptrs;
    ~DevMem() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <class T>
    cudaError_t alloc(T** out, size_t count) {
        void* p = nullptr;
        if (injected_alloc_failure()) return cudaErrorMemoryAllocation;
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(count * sizeof(T), 16));
        if (e != cudaSuccess) return e;
        ptrs.push_back(p);
        *out = static_cast<T*>(p);
        return cudaSuccess;
    }
};

template <class F>
void parallel_rows(size_t n, F&& f) {
    const size_t threads = std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), n / 65536 + 1));
    if (threads == 1) {
        f(size_t(0), n);
        return;
    }
    std::vector<std::thread> pool;
    for (size_t t = 0; t < threads; ++t) pool.emplace_back([&, t] { f(n * t / threads, n * (t + 1) / threads); });
    for (auto& th : pool) th.join();
}

uint32_t pow2_at_least(uint64_t x) {
    uint32_t p = 1;
    while (p < x && p < (1u << 30)) p <<= 1;
    return p;
}

}  // namespace

void gpu_build_defaults(GpuBuildOptions* o) { *o = GpuBuildOptions(); }

int gpu_link(HostIndex& ix, uint32_t first, int device, const GpuBuildOptions& opt, GpuBuildReport* rep) {
    const Params& P = ix.params;
    const size_t n64 = ix.node_count();
    if (rep) *rep = GpuBuildReport();
    if (first >= n64) return HNSW_OK;
    if (n64 >= (size_t(1) << 31)) return set_error(HNSW_ERR_INVALID_ARGUMENT, "device build: too many nodes");
    if (!(opt.wave_fraction > 0.0) || opt.wave_fraction > 1.0)
        return set_error(HNSW_ERR_INVALID_ARGUMENT, "device build: wave_fraction must be in (0, 1]");
    int ndev = 0;
    CU(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    if (device < 0 || device >= ndev) return set_error(HNSW_ERR_INVALID_ARGUMENT, "invalid device ordinal");
    CU(cudaSetDevice(device), "cudaSetDevice");
    const uint32_t n = uint32_t(n64);
    const uint32_t dim = ix.dim, dp = round_up(dim, 32);
    const uint32_t m = P.m, m0 = P.m0, mp = round_up(m, 32), m0p = round_up(m0, 32);
    const uint32_t capmax = std::max(m, m0);
    const uint32_t ef = std::max(P.ef_construction, m);

    // Upper-layer block offsets.
    std::vector<uint32_t> up_off(n);
    uint64_t blocks = 0;
    for (uint32_t i = 0; i < n; ++i) {
        up_off[i] = uint32_t(blocks);
        blocks += ix.levels[i];
    }
    if (n + blocks >= (uint64_t(1) << 32)) return set_error(HNSW_ERR_INVALID_ARGUMENT, "device build: too many lists");

    // Wave plan.
    std::vector<Wave> waves;
    bool has_entry = ix.has_entry();
    uint32_t entry = has_entry ? ix.entry_id() : 0, top = has_entry ? ix.top_level() : 0;
    uint32_t next = first;
    if (!has_entry) {
        entry = next;
        top = ix.levels[next];
        ++next;
    }
    uint32_t max_records = 0;
    const uint32_t max_wave = std::max<uint32_t>(1, opt.max_wave);
    while (next < n) {
        uint64_t w = uint64_t(std::floor(double(next) * opt.wave_fraction));
        w = std::max<uint64_t>(1, std::min<uint64_t>({w, max_wave, uint64_t(n - next)}));
        for (uint32_t j = next; j < next + w; ++j)
            if (ix.levels[j] > top) {
                w = j == next ? 1 : j - next;
                break;
            }
        uint64_t records = 0;
        for (uint32_t j = next; j < next + w; ++j) records += uint64_t(std::min<uint32_t>(ix.levels[j], top) + 1) * m;
        if (records >= (uint64_t(1) << 31))
            return set_error(HNSW_ERR_INVALID_ARGUMENT, "device build: wave too large");
        waves.push_back(Wave{next, uint32_t(w), entry, top, uint32_t(records)});
        max_records = std::max(max_records, uint32_t(records));
        if (w == 1 && ix.levels[next] > top) {
            entry = next;
            top = ix.levels[next];
        }
        next += uint32_t(w);
    }

    cudaDeviceProp prop;
    CU(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
    const uint32_t sms = uint32_t(prop.multiProcessorCount);
    const size_t optin = size_t(prop.sharedMemPerBlockOptin);
    const size_t budget = std::min<size_t>(optin, 220 * 1024);

    // Search geometry.
    BuildArgs a;
    a.selection = P.selection;
    a.extend = P.selection && P.extend_candidates;
    a.keep_pruned = P.keep_pruned;
    a.ef = ef;
    // The visited hash holds about 16 entries per unit of ef (a layer-0
    // search at ef = 200 visits 1-2k nodes); a search that passes 3/4 of it
    // continues in its HBM bitmap. After the search the hash region holds
    // the staged candidate rows of the selection and, when they fit in a
    // region of at most 24 KB, the selected rows.
    const size_t rowb = size_t(dp) * 4;
    a.hash_cap = opt.hash_cap ? std::max<uint32_t>(opt.hash_cap, 64)
                              : round_up(std::max<uint32_t>(1024, std::min<uint32_t>(16 * ef, 1u << 20)), 32);
    auto layout_region = [&]() {
        const size_t hb = size_t(a.hash_cap) * 4;
        const size_t want = size_t(m + 8) * rowb;
        if (want <= std::max<size_t>(hb, 24 * 1024)) {
            a.region_bytes = uint32_t(std::max(hb, want));
            a.sel_in_stage = 1;
            a.sel_rows = 0;
            a.stage_rows = uint32_t(std::min<size_t>(32, (a.region_bytes - size_t(m) * rowb) / rowb));
        } else {
            a.region_bytes = uint32_t(hb);
            a.sel_in_stage = 0;
            a.sel_rows = 0;
            a.stage_rows = uint32_t(std::min<size_t>(32, hb / rowb));
        }
        if (!opt.hash_cap) a.hash_cap = a.region_bytes / 4;
    };
    layout_region();
    size_t bytes = build_search_bytes(dp, ef, a.region_bytes, m, a.sel_rows);
    while (bytes > budget / 4 && a.hash_cap > 4096 && !opt.hash_cap) {
        a.hash_cap = round_up(a.hash_cap / 2, 32);
        layout_region();
        bytes = build_search_bytes(dp, ef, a.region_bytes, m, a.sel_rows);
    }
    const bool s_global = bytes > budget;
    if (s_global) {
        // cp.async stages into shared memory only: no staging from HBM scratch.
        a.stage_rows = 0;
        a.sel_in_stage = 0;
        bytes = build_search_bytes(dp, ef, a.region_bytes, m, a.sel_rows);
    }
    a.bytes_per_warp = uint32_t(bytes);
    uint32_t s_blocks_per_sm = 0;
    if (s_global) {
        a.warps_per_block = 4;
        s_blocks_per_sm = 2;
    } else {
        // Warps per block that maximise resident warps per SM.
        uint32_t best = 0;
        for (uint32_t wpb : {1u, 2u, 4u, 8u}) {
            if (size_t(a.bytes_per_warp) * wpb > budget) continue;
            int nb = 0;
            CU(gpu_build_occupancy(true, int(wpb) * 32, size_t(a.bytes_per_warp) * wpb, &nb),
               "occupancy (build search)");
            if (uint32_t(nb) * wpb > best) {
                best = uint32_t(nb) * wpb;
                a.warps_per_block = wpb;
                s_blocks_per_sm = uint32_t(nb);
            }
        }
        if (best == 0) {
            a.warps_per_block = 1;
            s_blocks_per_sm = 1;
        }
    }
    const uint32_t s_max_blocks = s_blocks_per_sm * sms;
    const uint32_t s_slots = s_max_blocks * a.warps_per_block;

    // Connect geometry.
    a.c_stage_rows = uint32_t(std::min<size_t>(capmax + 1, std::max<size_t>(1, 49152 / rowb)));
    a.c_sel_rows = (a.c_stage_rows < capmax + 1 && size_t(capmax) * rowb <= 32768) ? capmax : 0;
    size_t cbytes = build_connect_bytes(dp, capmax, a.c_stage_rows, a.c_sel_rows);
    const bool c_global = cbytes > budget;
    if (c_global) {
        a.c_stage_rows = 0;
        a.c_sel_rows = 0;
        cbytes = build_connect_bytes(dp, capmax, 0, 0);
    }
    a.c_bytes_per_warp = uint32_t(cbytes);
    uint32_t c_blocks_per_sm = 0;
    if (c_global) {
        a.c_warps_per_block = 4;
        c_blocks_per_sm = 2;
    } else {
        uint32_t best = 0;
        for (uint32_t wpb : {1u, 2u, 4u, 8u}) {
            if (size_t(a.c_bytes_per_warp) * wpb > budget) continue;
            int nb = 0;
            CU(gpu_build_occupancy(false, int(wpb) * 32, size_t(a.c_bytes_per_warp) * wpb, &nb),
               "occupancy (build connect)");
            if (uint32_t(nb) * wpb > best) {
                best = uint32_t(nb) * wpb;
                a.c_warps_per_block = wpb;
                c_blocks_per_sm = uint32_t(nb);
            }
        }
        if (best == 0) {
            a.c_warps_per_block = 1;
            c_blocks_per_sm = 1;
        }
    }
    const uint32_t c_max_blocks = c_blocks_per_sm * sms;
    const uint32_t c_slots = c_max_blocks * a.c_warps_per_block;

    // Device memory.
    DevMem mem;
    cudaStream_t stream = nullptr;
    CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() {
            if (s) cudaStreamDestroy(s);
        }
    } sg{stream};
    float* d_vec;
    uint8_t* d_levels;
    uint32_t *d_up, *d_adj0, *d_adjU;
    CU(mem.alloc(&d_vec, size_t(n) * dp), "cudaMalloc (vectors)");
    CU(mem.alloc(&d_levels, n), "cudaMalloc (levels)");
    CU(mem.alloc(&d_up, n), "cudaMalloc (up_off)");
    CU(mem.alloc(&d_adj0, size_t(n) * m0p), "cudaMalloc (layer 0)");
    CU(mem.alloc(&d_adjU, size_t(blocks) * mp), "cudaMalloc (upper layers)");
    const size_t nlists = size_t(n) + blocks;
    CU(mem.alloc(&a.cnt, nlists), "cudaMalloc (counts)");
    CU(mem.alloc(&a.base, nlists), "cudaMalloc (bases)");
    CU(mem.alloc(&a.rec, max_records), "cudaMalloc (records)");
    CU(mem.alloc(&a.touched, max_records), "cudaMalloc (touched)");
    CU(mem.alloc(&a.bkt, max_records), "cudaMalloc (buckets)");
    CU(mem.alloc(&a.wc, 1), "cudaMalloc (wave counters)");
    CU(mem.alloc(&a.totals, 1), "cudaMalloc (totals)");
    a.spill_words = round_up((n + 31) / 32, 4);
    CU(mem.alloc(&a.spill, size_t(s_slots) * a.spill_words), "cudaMalloc (spill bitmaps)");
    if (s_global) CU(mem.alloc(&a.gscratch, size_t(s_slots) * a.bytes_per_warp), "cudaMalloc (search scratch)");
    if (c_global) CU(mem.alloc(&a.c_gscratch, size_t(c_slots) * a.c_bytes_per_warp), "cudaMalloc (connect scratch)");
    if (a.extend) {
        a.ext_cap = std::max(ef, capmax + 1) * (capmax + 1);
        a.ext_hash_cap = pow2_at_least(2ull * a.ext_cap);
        const size_t slots = std::max(s_slots, c_slots);
        CU(mem.alloc(&a.ext, slots * a.ext_cap), "cudaMalloc (extension pools)");
        CU(mem.alloc(&a.ext_hash, slots * a.ext_hash_cap), "cudaMalloc (extension sets)");
        a.side_stride = capmax;
        CU(mem.alloc(&a.side, size_t(max_records) * a.side_stride), "cudaMalloc (side lists)");
    }
    a.max_records = max_records;
    CU(cudaMemsetAsync(a.cnt, 0, nlists * 4, stream), "cudaMemset (counts)");
    CU(cudaMemsetAsync(a.totals, 0, sizeof(BuildTotals), stream), "cudaMemset (totals)");
    CU(cudaMemsetAsync(a.spill, 0, size_t(s_slots) * a.spill_words * 4, stream), "cudaMemset (spill)");

    // Upload: vectors (rows padded with zeros), levels, offsets, lists.
    if (dp == dim) {
        CU(cudaMemcpyAsync(d_vec, ix.vectors.data(), size_t(n) * dim * 4, cudaMemcpyHostToDevice, stream),
           "cudaMemcpy (vectors)");
    } else {
        CU(cudaMemsetAsync(d_vec, 0, size_t(n) * dp * 4, stream), "cudaMemset (vectors)");
        CU(cudaMemcpy2DAsync(d_vec, size_t(dp) * 4, ix.vectors.data(), size_t(dim) * 4, size_t(dim) * 4, n,
                             cudaMemcpyHostToDevice, stream),
           "cudaMemcpy2D (vectors)");
    }
    CU(cudaMemcpyAsync(d_levels, ix.levels.data(), n, cudaMemcpyHostToDevice, stream), "cudaMemcpy (levels)");
    CU(cudaMemcpyAsync(d_up, up_off.data(), size_t(n) * 4, cudaMemcpyHostToDevice, stream), "cudaMemcpy (up_off)");
    std::vector<uint32_t> h0(size_t(n) * m0p), hU(size_t(blocks) * mp);
    parallel_rows(n, [&](size_t b, size_t e) {
        for (size_t i = b; i < e; ++i) {
            const uint32_t* blk = ix.block(uint32_t(i), 0);
            const uint32_t c = std::min(blk[0], m0);
            uint32_t* out = h0.data() + i * m0p;
            std::memcpy(out, blk + 1, size_t(c) * 4);
            std::fill(out + c, out + m0p, kSentinel);
            for (uint32_t l = 1; l <= ix.levels[i]; ++l) {
                const uint32_t* ub = ix.block(uint32_t(i), l);
                const uint32_t cu = std::min(ub[0], m);
                uint32_t* uo = hU.data() + (size_t(up_off[i]) + l - 1) * mp;
                std::memcpy(uo, ub + 1, size_t(cu) * 4);
                std::fill(uo + cu, uo + mp, kSentinel);
            }
        }
    });
    CU(cudaMemcpyAsync(d_adj0, h0.data(), h0.size() * 4, cudaMemcpyHostToDevice, stream), "cudaMemcpy (layer 0)");
    if (blocks)
        CU(cudaMemcpyAsync(d_adjU, hU.data(), hU.size() * 4, cudaMemcpyHostToDevice, stream),
           "cudaMemcpy (upper layers)");

    a.g.n = n;
    a.g.dim = dim;
    a.g.dp = dp;
    a.g.m = m;
    a.g.m0 = m0;
    a.g.mp = mp;
    a.g.m0p = m0p;
    a.g.metric = ix.metric;
    a.g.vec = d_vec;
    a.g.adj0 = d_adj0;
    a.g.up_off = d_up;
    a.g.adjU = d_adjU;
    a.g.levels = d_levels;

    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    CU(cudaEventCreate(&ev0), "cudaEventCreate");
    CU(cudaEventCreate(&ev1), "cudaEventCreate");
    struct EventGuard {
        cudaEvent_t a, b;
        ~EventGuard() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } eg{ev0, ev1};
    // Per-phase timing: events after each search step and each connect
    // step (only when asked; they are recorded on the same stream).
    std::vector<cudaEvent_t> marks;
    struct MarkGuard {
        std::vector<cudaEvent_t>& v;
        ~MarkGuard() {
            for (cudaEvent_t e : v) cudaEventDestroy(e);
        }
    } mg{marks};
    if (opt.timing) {
        marks.resize(2 * waves.size());
        for (auto& e : marks) CU(cudaEventCreate(&e), "cudaEventCreate");
    }
    TraceRange trace("hnsw.build_waves");
    CU(cudaEventRecord(ev0, stream), "cudaEventRecord");
    for (size_t i = 0; i < waves.size(); ++i) {
        const Wave& wv = waves[i];
        a.first = wv.first;
        a.count = wv.count;
        a.entry = wv.entry;
        a.top = wv.top;
        const uint32_t sb = std::min(s_max_blocks, (wv.count + a.warps_per_block - 1) / a.warps_per_block);
        const uint32_t cb = std::min(c_max_blocks, (wv.records + a.c_warps_per_block - 1) / a.c_warps_per_block);
        const uint32_t small = std::min<uint32_t>(4 * sms, wv.records / 256 + 1);
        CU(launch_build_search(a, std::max(1u, sb), stream), "device build (search)");
        if (opt.timing) CU(cudaEventRecord(marks[2 * i], stream), "cudaEventRecord");
        CU(launch_build_connect(a, std::max(1u, cb), small, stream), "device build (connect)");
        if (opt.timing) CU(cudaEventRecord(marks[2 * i + 1], stream), "cudaEventRecord");
    }
    CU(cudaEventRecord(ev1, stream), "cudaEventRecord");
    CU(cudaStreamSynchronize(stream), "device build");
    float ms = 0.0f;
    CU(cudaEventElapsedTime(&ms, ev0, ev1), "cudaEventElapsedTime");
    double search_ms = 0.0, connect_ms = 0.0;
    for (size_t i = 0; opt.timing && i < waves.size(); ++i) {
        float t0 = 0.0f, t1 = 0.0f;
        CU(cudaEventElapsedTime(&t0, i ? marks[2 * i - 1] : ev0, marks[2 * i]), "cudaEventElapsedTime");
        CU(cudaEventElapsedTime(&t1, marks[2 * i], marks[2 * i + 1]), "cudaEventElapsedTime");
        search_ms += t0;
        connect_ms += t1;
    }
    BuildTotals tot;
    CU(cudaMemcpy(&tot, a.totals, sizeof(tot), cudaMemcpyDeviceToHost), "cudaMemcpy (totals)");
    CU(cudaMemcpy(h0.data(), d_adj0, h0.size() * 4, cudaMemcpyDeviceToHost), "cudaMemcpy (layer 0 back)");
    if (blocks)
        CU(cudaMemcpy(hU.data(), d_adjU, hU.size() * 4, cudaMemcpyDeviceToHost), "cudaMemcpy (upper layers back)");

    // Write the lists back (count word, then the ids).
    parallel_rows(n, [&](size_t b, size_t e) {
        for (size_t i = b; i < e; ++i) {
            uint32_t* blk = ix.block(uint32_t(i), 0);
            const uint32_t* in = h0.data() + i * m0p;
            uint32_t c = 0;
            while (c < m0 && in[c] != kSentinel) ++c;
            blk[0] = c;
            std::memcpy(blk + 1, in, size_t(c) * 4);
            for (uint32_t l = 1; l <= ix.levels[i]; ++l) {
                uint32_t* ub = ix.block(uint32_t(i), l);
                const uint32_t* ui = hU.data() + (size_t(up_off[i]) + l - 1) * mp;
                uint32_t cu = 0;
                while (cu < m && ui[cu] != kSentinel) ++cu;
                ub[0] = cu;
                std::memcpy(ub + 1, ui, size_t(cu) * 4);
            }
        }
    });
    ix.entry_word = (uint64_t(top) << 32) | entry;
    if (rep) {
        rep->waves = uint32_t(waves.size());
        rep->nodes = n - first;
        rep->spills = tot.spills;
        rep->inexact = tot.inexact;
        rep->shrinks = tot.shrinks;
        rep->records = tot.records;
        rep->device_ms = ms;
        rep->search_ms = search_ms;
        rep->connect_ms = connect_ms;
        rep->dist_search = tot.dist_search;
        rep->dist_select = tot.dist_select;
        rep->dist_connect = tot.dist_connect;
        rep->lists0 = tot.lists0;
        rep->listsU = tot.listsU;
        rep->search_warps_per_block = a.warps_per_block;
        rep->search_blocks_per_sm = s_blocks_per_sm;
        rep->connect_warps_per_block = a.c_warps_per_block;
        rep->connect_blocks_per_sm = c_blocks_per_sm;
        rep->hash_cap = a.hash_cap;
    }
    return HNSW_OK;
}

}  // namespace hnswgpu
