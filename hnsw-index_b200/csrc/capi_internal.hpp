// Internals of the C ABI shared by capi.cpp and server.cpp: device buffers,
// per-call scratch slots, the index and brute-force handles, and the launch
// helper of one search.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <functional>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "brute_tc.hpp"
#include "device.hpp"
#include "hnsw_gpu.h"
#include "host_index.hpp"

namespace hnswgpu {

// Records the message of the last failure on this thread; returns status.
int set_error(int status, const std::string& msg);
const char* last_error_text();
int from_err(const Err& e);
int cuda_fail(cudaError_t e, const char* where);

#define CU(call, where)                                      \
    do {                                                     \
        cudaError_t _e = (call);                             \
        if (_e != cudaSuccess) return ::hnswgpu::cuda_fail(_e, where); \
    } while (0)

inline uint32_t round_up(uint32_t x, uint32_t a) { return (x + a - 1) / a * a; }

// Device allocations still to fail on purpose (hnsw_gpu_debug_fail_allocations):
// a host-side test hook for the out-of-device-memory paths.
inline std::atomic<int> g_fail_allocations{0};
// Visited-hash tags (hnsw_gpu_debug_visit_tags): 0 automatic, -1 off (32-bit
// ids), k > 0 an id space of at least k bits.
inline std::atomic<int> g_visit_tag_bits{0};
inline bool injected_alloc_failure() {
    int n = g_fail_allocations.load(std::memory_order_relaxed);
    while (n > 0)
        if (g_fail_allocations.compare_exchange_weak(n, n - 1, std::memory_order_relaxed)) return true;
    return false;
}

// Growable device buffer.
struct DBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t need) {
        if (need <= bytes) return cudaSuccess;
        if (injected_alloc_failure()) return cudaErrorMemoryAllocation;  // buffer left as it was
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, need);
        if (e == cudaSuccess) bytes = need;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

// One concurrent call's stream and scratch.
struct Slot {
    cudaStream_t stream = nullptr;
    DBuf q, ks, efs, fbits, fused, fids, okeys, odist, ocount, ostatus, work, overflow, counters;
    DBuf g_results, g_cands, g_visited;
    uint32_t g_warps = 0, g_ef_cap = 0, g_cand_cap = 0;
    uint64_t g_words = 0;
    DBuf spill_bits, spill_cands;  // persistent-mode spill areas (bitmaps kept zero)
    DBuf cold_pool, cold_tab; // cold candidate lists (persistent and retry warps)
    DBuf last_pool, last_tab, overflow2;  // last-resort pass (private cold regions)
    DBuf planned;                         // selectivity planner flags
    size_t last_nq = 0;
    ~Slot() {
        for (DBuf* b : {&q, &ks, &efs, &fbits, &fused, &fids, &okeys, &odist, &ocount, &ostatus, &work, &overflow, &counters,
                        &g_results, &g_cands, &g_visited, &spill_bits, &spill_cands, &cold_pool, &cold_tab, &last_pool,
                        &last_tab, &overflow2, &planned})
            b->release();
        if (stream) cudaStreamDestroy(stream);
    }
};

struct SlotPool {
    std::mutex mu;
    std::vector<std::unique_ptr<Slot>> free;
    int device = 0;
    int acquire(Slot** out) {
        {
            std::lock_guard<std::mutex> g(mu);
            if (!free.empty()) {
                *out = free.back().release();
                free.pop_back();
                return HNSW_OK;
            }
        }
        auto* s = new (std::nothrow) Slot();
        if (!s) return set_error(HNSW_ERR_INVALID_ARGUMENT, "out of host memory");
        cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete s;
            return cuda_fail(e, "cudaStreamCreate");
        }
        *out = s;
        return HNSW_OK;
    }
    void release(Slot* s) {
        std::lock_guard<std::mutex> g(mu);
        free.emplace_back(s);
    }
};

// A named range on the NVTX timeline around a host-side phase (staging,
// enqueue, copies, a build wave). Profilers that attach an NVTX tool (Nsight
// Systems, Nsight Compute with --nvtx) show it; without one it costs a
// function call.
struct TraceRange {
    explicit TraceRange(const char* name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange&) = delete;
    TraceRange& operator=(const TraceRange&) = delete;
};

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// Scratch geometry per (ef bound): results, candidates and the visited
// hash sized so that a typical traversal at that ef stays in shared memory.
// Queries whose ef exceeds the fast kernel's 1024 go to the retry pass.
SearchGeometry pick_geometry(uint32_t ef_max, uint32_t dp, uint32_t dc, bool persistent, bool filtered, uint32_t n);

}  // namespace hnswgpu

// The handle types of the C ABI (opaque to callers).
using hnswgpu::DBuf;
using hnswgpu::DeviceGuard;
using hnswgpu::DeviceIndexView;
using hnswgpu::Slot;
using hnswgpu::SlotPool;
using hnswgpu::Builder;

struct hnsw_gpu_index {
    int device = 0;
    int num_sms = 148;
    hnsw_index_info info{};
    DeviceIndexView view;
    DBuf vec, codes, norms, offset, adj0, upoff, adjU, keys, dead;
    SlotPool slots;
    bool counters = false;
    std::mutex counters_mu;
    std::vector<uint32_t> last_counters;
    // Scratch of the device-pointer entry point: one slot, ordered on the
    // device (an event joins each call after the previous one).
    std::mutex dev_mu;
    std::unique_ptr<Slot> dev_slot;
    // Fixed schedule (hnsw_gpu_set_schedule); ef_cap == 0 means automatic.
    hnswgpu::SearchGeometry fixed{0, 0, 0, 0, 0};
    // Autotuned schedules (hnsw_gpu_autotune) per ef bucket, bucket b
    // covering max(ef, k) in (32(b-1), 32b], b = 1..32 (the last one also
    // everything above 1024), one per mode; ef_cap == 0 means not tuned.
    // `mode` is the faster mode of the bucket (-1: not tuned).
    struct Tuned {
        hnswgpu::SearchGeometry geo[2] = {{0, 0, 0, 0, 0}, {0, 0, 0, 0, 0}};
        int32_t mode = -1;
    };
    std::mutex tune_mu;
    Tuned tuned[33];
    cudaEvent_t dev_done = nullptr;
    // Tensor-core traversal rows, built on first use (tc_mu): BF16 high
    // parts, low parts (BF16X3), f32 squared norms (L2).
    std::mutex tc_mu;
    DBuf tc_hi, tc_lo, tc_norm;
    DBuf chk;  // bounds-check word of the checked build (2 x u32)
    bool tc_hi_ready = false, tc_lo_ready = false;
    ~hnsw_gpu_index() {
        DeviceGuard g(device);
        if (dev_done) {
            cudaEventSynchronize(dev_done);
            cudaEventDestroy(dev_done);
        }
        dev_slot.reset();
        for (DBuf* b : {&vec, &codes, &norms, &offset, &adj0, &upoff, &adjU, &keys, &dead, &tc_hi, &tc_lo, &tc_norm, &chk})
            b->release();
        std::lock_guard<std::mutex> l(slots.mu);
        slots.free.clear();
    }
};

struct hnsw_gpu_brute {
    int device = 0;
    int num_sms = 148;
    uint32_t n = 0, dim = 0, dp = 0;
    int metric = 0;
    float max_xnorm = 0.0f;  // largest row norm (error margins of the tensor-core path)
    DBuf base, keys;
    SlotPool slots;
    std::mutex mu;
    DBuf qprep, part, okeys, odist, ocount, ostatus, q;
    DBuf fbits, fused, fids;  // filter bitmaps, flags and bitmap ids of a filtered search
    // Tensor-core path: BF16 operand rows per term count (index 0: 1 term, 1: 3 terms).
    DBuf bop[2], xnorm2;
    uint32_t bop_kp[2] = {0, 0};
    DBuf aop, dense, thr1, thr2, margin, qnorm2, ccount, cand, err;
    uint64_t last_candidates = 0, last_queries = 0;
    float last_ms[4] = {0, 0, 0, 0};
    long long wait_budget = 4000000000ll;  // tensor-core pipeline waits, clock cycles
    uint32_t stall = 0;                    // test switch: the MMA issuer's wait runs out
    uint32_t tc_pairs = 0;                 // paired (cta_group::2) tensor-core kernel
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    cudaStream_t stream = nullptr;
    ~hnsw_gpu_brute() {
        DeviceGuard g(device);
        for (DBuf* b : {&base, &keys, &qprep, &part, &okeys, &odist, &ocount, &ostatus, &q, &fbits, &fused, &fids,
                        &bop[0], &bop[1], &xnorm2,
                        &aop, &dense, &thr1, &thr2, &margin, &qnorm2, &ccount, &cand, &err})
            b->release();
        for (cudaEvent_t& e : ev)
            if (e) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
    }
};

struct hnsw_builder {
    std::unique_ptr<Builder> b;
    hnsw_gpu_build_stats last{};  // figures of the last device link
};

namespace hnswgpu {
// Enqueues one search on `stream` with device pointers. ef_max bounds every
// per-query max(ef, k) of the batch.
int enqueue_search(hnsw_gpu_index* gi, Slot* s, const float* d_q, size_t nq, const hnsw_search_opts& o,
                   const uint32_t* d_ks, const uint32_t* d_efs, const uint64_t* d_fbits, const uint8_t* d_fused,
                   const uint32_t* d_fids, uint64_t* d_keys, float* d_dist, uint32_t* d_count, int32_t* d_status, uint32_t ef_max,
                   uint32_t out_stride, cudaStream_t stream, const SearchGeometry* force = nullptr,
                   bool publish = false);
// The ef bucket of the tuning table for a batch whose max(ef, k) is ef_max.
inline uint32_t tune_bucket(uint32_t ef_max) {
    return ef_max > 1024 ? 32u : std::max<uint32_t>(1, (ef_max + 31) / 32);
}
}  // namespace hnswgpu
