// Request loop over a resident device index: continuous batching with
// admission by device scratch.
//
// Callers submit single searches (query, k, ef, optional key filter). A
// dispatcher thread forms batches from the pending queue and launches each on
// its own stream as soon as one of the batch slots (device scratch for one
// launch: staging, outputs, spill areas) is free, so requests that arrive
// while earlier batches run are admitted and their work overlaps on the
// device. When every slot is busy, requests wait on the host; when the
// pending queue is full, submission is rejected (ADMISSION_REJECTED). A batch
// runs the persistent search kernel with per-query k, ef and filters, so each
// result equals the result of the same search run alone. The kernel writes
// each query's results into mapped host memory and publishes its status last,
// so a request completes when its own query does, not when its batch does.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <thread>

#include "capi_internal.hpp"

using namespace hnswgpu;

namespace {

using Clock = std::chrono::steady_clock;

double now_us() {
    return std::chrono::duration<double, std::micro>(Clock::now().time_since_epoch()).count();
}

enum class ReqState : uint8_t { Free, Pending, Inflight, Done };

struct Request {
    ReqState state = ReqState::Free;
    uint32_t k = 0, ef = 0;
    int32_t filter_id = -1;
    int32_t status = 0;
    uint32_t count = 0;
    double t_arrival = 0, t_done = 0;
    uint64_t ticket = 0;
    bool cancelled = false;  // in flight when cancelled: its results are discarded
};

// Host staging of one batch (pinned) plus its device scratch slot.
struct BatchSlot {
    Slot* slot = nullptr;
    cudaEvent_t done = nullptr;
    bool busy = false;
    std::vector<uint64_t> tickets;
    float* h_q = nullptr;
    uint32_t* h_ks = nullptr;
    uint32_t* h_efs = nullptr;
    uint8_t* h_fused = nullptr;
    uint32_t* h_fids = nullptr;
    // Outputs, mapped into the device address space (the kernel writes them).
    uint64_t* h_keys = nullptr;
    float* h_dist = nullptr;
    uint32_t* h_count = nullptr;
    int32_t* h_status = nullptr;
    uint64_t* d_keys = nullptr;
    float* d_dist = nullptr;
    uint32_t* d_count = nullptr;
    int32_t* d_status = nullptr;
    std::vector<uint8_t> finished;  // per batch entry: request already completed
    uint32_t remaining = 0;
};

// Status value of an entry whose query has not published yet.
constexpr int32_t kUnpublished = -1;
// Status the fast kernels write before the retry passes take a query over.
constexpr int32_t kRetrying = HNSW_ERR_SCRATCH_OVERFLOW;

}  // namespace

struct hnsw_gpu_server {
    hnsw_gpu_index* index = nullptr;
    hnsw_server_config cfg{};
    uint32_t dim = 0, words = 0;
    std::vector<Request> req;
    std::vector<float> q;            // cap x dim
    DBuf bank;                       // filter bank on the device
    std::vector<uint64_t> keys;      // cap x max_k
    std::vector<float> dist;         // cap x max_k
    uint64_t cap = 0;
    uint64_t next_ticket = 1;
    std::deque<uint64_t> pending;
    std::vector<BatchSlot> batches;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::atomic<bool> stop{false};
    std::thread dispatcher;
    int error = HNSW_OK;
    uint64_t launched_batches = 0, launched_queries = 0;

    Request& at(uint64_t ticket) { return req[ticket % cap]; }
};

namespace {

int stage_and_launch(hnsw_gpu_server* s, BatchSlot& b, std::vector<uint64_t>& tickets) {
    TraceRange trace("hnsw.server_batch");
    const uint32_t n = uint32_t(tickets.size());
    const uint32_t dim = s->dim, K = s->cfg.max_k;
    bool any_filter = false;
    uint32_t ef_max = 1;
    for (uint32_t i = 0; i < n; ++i) {
        Request& r = s->at(tickets[i]);
        std::memcpy(b.h_q + size_t(i) * dim, &s->q[(tickets[i] % s->cap) * dim], size_t(dim) * 4);
        b.h_ks[i] = r.k;
        b.h_efs[i] = r.ef;
        b.h_status[i] = kUnpublished;
        ef_max = std::max(ef_max, std::max(r.k, r.ef));
        b.h_fused[i] = r.filter_id >= 0 ? 1 : 0;
        b.h_fids[i] = r.filter_id >= 0 ? uint32_t(r.filter_id) : 0u;
        any_filter |= r.filter_id >= 0;
    }
    Slot* sl = b.slot;
    cudaStream_t st = sl->stream;
    CU(sl->q.ensure(size_t(s->cfg.max_batch) * dim * 4), "server queries");
    CU(sl->ks.ensure(size_t(s->cfg.max_batch) * 4), "server ks");
    CU(sl->efs.ensure(size_t(s->cfg.max_batch) * 4), "server efs");
    CU(cudaMemcpyAsync(sl->q.p, b.h_q, size_t(n) * dim * 4, cudaMemcpyHostToDevice, st), "copy queries");
    CU(cudaMemcpyAsync(sl->ks.p, b.h_ks, size_t(n) * 4, cudaMemcpyHostToDevice, st), "copy ks");
    CU(cudaMemcpyAsync(sl->efs.p, b.h_efs, size_t(n) * 4, cudaMemcpyHostToDevice, st), "copy efs");
    const uint64_t* d_fb = nullptr;
    const uint8_t* d_fu = nullptr;
    const uint32_t* d_fi = nullptr;
    if (any_filter && s->words) {
        CU(sl->fused.ensure(size_t(s->cfg.max_batch)), "server filter flags");
        CU(sl->fids.ensure(size_t(s->cfg.max_batch) * 4), "server filter ids");
        CU(cudaMemcpyAsync(sl->fused.p, b.h_fused, n, cudaMemcpyHostToDevice, st), "copy filter flags");
        CU(cudaMemcpyAsync(sl->fids.p, b.h_fids, size_t(n) * 4, cudaMemcpyHostToDevice, st), "copy filter ids");
        d_fb = s->bank.as<uint64_t>();
        d_fu = sl->fused.as<uint8_t>();
        d_fi = sl->fids.as<uint32_t>();
    }
    hnsw_search_opts o{};
    o.k = K;
    o.ef = s->cfg.max_ef;
    o.quantized = s->cfg.quantized;
    o.filter_nbits = s->cfg.filter_nbits;
    o.filter_by_node = s->cfg.filter_by_node;
    o.filter_stride = s->words;
    o.out_stride = K;
    o.mode = s->cfg.mode;
    b.finished.assign(n, 0);
    b.remaining = n;
    // Scratch sized for the batch's own largest max(ef, k).
    int r = enqueue_search(s->index, sl, sl->q.as<float>(), n, o, sl->ks.as<uint32_t>(), sl->efs.as<uint32_t>(), d_fb,
                           d_fu, d_fi, b.d_keys, b.d_dist, b.d_count, b.d_status, ef_max, K, st, nullptr, true);
    if (r != HNSW_OK) return r;
    CU(cudaEventRecord(b.done, st), "record batch event");
    return HNSW_OK;
}

// Moves entry i of a batch into the request table (caller holds mu).
void complete_one(hnsw_gpu_server* s, BatchSlot& b, size_t i, int32_t status, double t) {
    const uint32_t K = s->cfg.max_k;
    Request& r = s->at(b.tickets[i]);
    const uint64_t row = b.tickets[i] % s->cap;
    r.status = r.cancelled ? HNSW_ERR_CANCELLED : status;
    r.count = r.status == 0 ? std::min(b.h_count[i], r.k) : 0;
    std::memcpy(&s->keys[row * K], b.h_keys + i * K, size_t(r.count) * 8);
    std::memcpy(&s->dist[row * K], b.h_dist + i * K, size_t(r.count) * 4);
    r.t_done = t;
    r.state = ReqState::Done;
    b.finished[i] = 1;
    --b.remaining;
}

// Completes the entries whose queries have published; with `all` (the
// batch's event has fired) every entry. Returns whether any completed.
bool harvest(hnsw_gpu_server* s, BatchSlot& b, bool all) {
    const double t = now_us();
    bool any = false;
    for (size_t i = 0; i < b.tickets.size() && b.remaining; ++i) {
        if (b.finished[i]) continue;
        const int32_t st = reinterpret_cast<volatile int32_t*>(b.h_status)[i];
        if (!all && (st == kUnpublished || st == kRetrying)) continue;
        std::atomic_thread_fence(std::memory_order_acquire);
        complete_one(s, b, i, st, t);
        any = true;
    }
    if (all) {
        b.tickets.clear();
        b.busy = false;
    }
    return any;
}

void dispatch_loop(hnsw_gpu_server* s) {
    DeviceGuard dg(s->index->device);
    std::vector<uint64_t> take;
    while (true) {
        std::unique_lock<std::mutex> lock(s->mu);
        // Retire finished batches.
        bool retired = false;
        int inflight = 0;
        for (BatchSlot& b : s->batches) {
            if (!b.busy) continue;
            if (cudaEventQuery(b.done) == cudaSuccess) {
                harvest(s, b, true);
                retired = true;
            } else {
                retired |= harvest(s, b, false);
                ++inflight;
            }
        }
        if (retired) s->cv_done.notify_all();
        if (s->stop && s->pending.empty() && inflight == 0) break;
        // Launch while a slot is free and work is waiting. With batches in
        // flight, a partial batch lingers briefly to gather more requests.
        BatchSlot* free_slot = nullptr;
        for (BatchSlot& b : s->batches)
            if (!b.busy) {
                free_slot = &b;
                break;
            }
        bool launch = false;
        if (free_slot && !s->pending.empty()) {
            const double oldest = s->at(s->pending.front()).t_arrival;
            launch = inflight == 0 || s->pending.size() >= s->cfg.max_batch ||
                     now_us() - oldest >= double(s->cfg.linger_us) || s->stop;
        }
        if (launch) {
            take.clear();
            while (!s->pending.empty() && take.size() < s->cfg.max_batch) {
                const uint64_t t = s->pending.front();
                s->pending.pop_front();
                s->at(t).state = ReqState::Inflight;
                take.push_back(t);
            }
            free_slot->busy = true;
            free_slot->tickets = take;
            const int r = stage_and_launch(s, *free_slot, free_slot->tickets);
            ++s->launched_batches;
            s->launched_queries += take.size();
            if (r != HNSW_OK) {
                s->error = r;
                for (uint64_t t : take) {
                    Request& q = s->at(t);
                    q.status = r;
                    q.count = 0;
                    q.t_done = now_us();
                    q.state = ReqState::Done;
                }
                free_slot->busy = false;
                free_slot->tickets.clear();
                s->cv_done.notify_all();
            }
            continue;
        }
        // Nothing to launch now: wait for a request, or poll the GPU.
        if (inflight == 0 && s->pending.empty()) {
            s->cv_work.wait_for(lock, std::chrono::milliseconds(5));
        } else {
            lock.unlock();
            std::this_thread::sleep_for(std::chrono::microseconds(inflight ? 10 : 5));
        }
    }
}

}  // namespace

extern "C" {

void hnsw_server_config_default(hnsw_server_config* c) {
    std::memset(c, 0, sizeof *c);
    c->max_batch = 2048;
    c->max_inflight = 4;
    c->max_pending = 1u << 16;
    c->max_k = 100;
    c->max_ef = 512;
    c->linger_us = 100;
    c->filter_nbits = 0;
    c->quantized = 0;
    c->filter_bank = nullptr;
    c->filter_count = 0;
    c->mode = HNSW_MODE_PERSISTENT;
}

int hnsw_gpu_server_start(hnsw_gpu_index* index, const hnsw_server_config* cfg_in, hnsw_gpu_server** out) {
    if (!index || !out) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    hnsw_server_config cfg;
    if (cfg_in) cfg = *cfg_in;
    else hnsw_server_config_default(&cfg);
    if (cfg.max_batch == 0 || cfg.max_inflight == 0 || cfg.max_pending == 0 || cfg.max_k == 0 || cfg.max_ef == 0 ||
        cfg.max_batch > (1u << 20) || cfg.max_inflight > 64 || cfg.max_k > 1024 || cfg.max_ef > 65536 ||
        (cfg.mode != HNSW_MODE_PLAIN && cfg.mode != HNSW_MODE_PERSISTENT && cfg.mode != HNSW_MODE_AUTO))
        return set_error(HNSW_ERR_INVALID_ARGUMENT, "server configuration out of range");
    if (cfg.quantized && !index->view.quantized)
        return set_error(HNSW_ERR_QUANTIZATION_DISABLED, "quantized search requested but quantization is not enabled");
    DeviceGuard dg(index->device);
    std::unique_ptr<hnsw_gpu_server> s(new hnsw_gpu_server());
    s->index = index;
    s->cfg = cfg;
    s->dim = index->view.dim;
    s->words = uint32_t((cfg.filter_nbits + 63) / 64);
    s->cap = uint64_t(cfg.max_pending) + uint64_t(cfg.max_inflight) * cfg.max_batch;
    if ((cfg.filter_count > 0) != (cfg.filter_bank != nullptr) || (cfg.filter_count && !s->words))
        return set_error(HNSW_ERR_INVALID_ARGUMENT, "filter bank needs filter_nbits, bitmaps and their count");
    s->req.resize(s->cap);
    s->q.resize(s->cap * s->dim);
    if (cfg.filter_count) {
        const size_t bytes = size_t(cfg.filter_count) * s->words * 8;
        CU(s->bank.ensure(bytes), "cudaMalloc filter bank");
        CU(cudaMemcpy(s->bank.p, cfg.filter_bank, bytes, cudaMemcpyHostToDevice), "copy filter bank");
    }
    s->cfg.filter_bank = nullptr;
    s->keys.resize(s->cap * cfg.max_k);
    s->dist.resize(s->cap * cfg.max_k);
    s->batches.resize(cfg.max_inflight);
    for (BatchSlot& b : s->batches) {
        int r = index->slots.acquire(&b.slot);
        if (r != HNSW_OK) return r;
        CU(cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming), "server event");
        const size_t B = cfg.max_batch;
        CU(cudaMallocHost(&b.h_q, B * s->dim * 4), "pinned queries");
        CU(cudaMallocHost(&b.h_ks, B * 4), "pinned ks");
        CU(cudaMallocHost(&b.h_efs, B * 4), "pinned efs");
        CU(cudaMallocHost(&b.h_fused, B), "pinned filter flags");
        CU(cudaMallocHost(&b.h_fids, B * 4), "pinned filter ids");
        CU(cudaHostAlloc(&b.h_keys, B * cfg.max_k * 8, cudaHostAllocMapped), "mapped keys");
        CU(cudaHostAlloc(&b.h_dist, B * cfg.max_k * 4, cudaHostAllocMapped), "mapped dist");
        CU(cudaHostAlloc(&b.h_count, B * 4, cudaHostAllocMapped), "mapped counts");
        CU(cudaHostAlloc(&b.h_status, B * 4, cudaHostAllocMapped), "mapped statuses");
        CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&b.d_keys), b.h_keys, 0), "mapped keys");
        CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&b.d_dist), b.h_dist, 0), "mapped dist");
        CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&b.d_count), b.h_count, 0), "mapped counts");
        CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&b.d_status), b.h_status, 0), "mapped statuses");
    }
    hnsw_gpu_server* raw = s.get();
    raw->dispatcher = std::thread(dispatch_loop, raw);
    *out = s.release();
    return HNSW_OK;
}

void hnsw_gpu_server_stop(hnsw_gpu_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->dispatcher.joinable()) s->dispatcher.join();
    DeviceGuard dg(s->index->device);
    for (BatchSlot& b : s->batches) {
        if (b.done) cudaEventDestroy(b.done);
        for (void* p : {(void*)b.h_q, (void*)b.h_ks, (void*)b.h_efs, (void*)b.h_fused, (void*)b.h_fids,
                        (void*)b.h_keys, (void*)b.h_dist, (void*)b.h_count, (void*)b.h_status})
            if (p) cudaFreeHost(p);
        if (b.slot) s->index->slots.release(b.slot);
    }
    s->bank.release();
    delete s;
}

// Admits requests whose arrival time (microseconds on the server clock, or
// now when arrival_us < 0) is given; the caller holds no lock.
static int submit_locked(hnsw_gpu_server* s, const float* query, uint32_t k, uint32_t ef, int32_t filter_id,
                         double arrival_us, uint64_t* ticket) {
    if (k == 0 || k > s->cfg.max_k || ef > s->cfg.max_ef)
        return set_error(HNSW_ERR_INVALID_ARGUMENT, "k or ef outside the server's bounds");
    if (filter_id >= 0 && uint32_t(filter_id) >= s->cfg.filter_count)
        return set_error(HNSW_ERR_INVALID_ARGUMENT, "filter id outside the server's filter bank");
    if (s->pending.size() >= s->cfg.max_pending)
        return set_error(HNSW_ERR_ADMISSION_REJECTED, "request queue full");
    const uint64_t t = s->next_ticket;
    Request& r = s->at(t);
    if (r.state != ReqState::Free) return set_error(HNSW_ERR_ADMISSION_REJECTED, "no free request slot");
    ++s->next_ticket;
    r.state = ReqState::Pending;
    r.ticket = t;
    r.k = k;
    r.ef = ef;
    r.filter_id = filter_id;
    r.status = 0;
    r.count = 0;
    r.cancelled = false;
    r.t_arrival = arrival_us >= 0 ? arrival_us : now_us();
    std::memcpy(&s->q[(t % s->cap) * s->dim], query, size_t(s->dim) * 4);
    s->pending.push_back(t);
    *ticket = t;
    return HNSW_OK;
}

int hnsw_gpu_submit(hnsw_gpu_server* s, const float* query, uint32_t k, uint32_t ef, int32_t filter_id,
                    uint64_t* ticket) {
    if (!s || !query || !ticket) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    int r;
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (s->stop) return set_error(HNSW_ERR_INVALID_ARGUMENT, "server stopped");
        r = submit_locked(s, query, k, ef, filter_id, -1.0, ticket);
    }
    if (r == HNSW_OK) s->cv_work.notify_one();
    return r;
}

int hnsw_gpu_cancel(hnsw_gpu_server* s, uint64_t ticket, int* cancelled) {
    if (!s || !cancelled) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> g(s->mu);
    Request& r = s->at(ticket);
    if (r.ticket != ticket || r.state == ReqState::Free) return set_error(HNSW_ERR_INVALID_ARGUMENT, "unknown ticket");
    *cancelled = 0;
    if (r.state == ReqState::Pending) {
        auto it = std::find(s->pending.begin(), s->pending.end(), ticket);
        if (it != s->pending.end()) s->pending.erase(it);
        r.status = HNSW_ERR_CANCELLED;
        r.count = 0;
        r.t_done = now_us();
        r.state = ReqState::Done;
        *cancelled = 1;
        s->cv_done.notify_all();
    } else if (r.state == ReqState::Inflight) {
        r.cancelled = true;
        *cancelled = 1;
    }
    return HNSW_OK;
}

int hnsw_gpu_poll(hnsw_gpu_server* s, uint64_t ticket, int* done) {
    if (!s || !done) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> g(s->mu);
    Request& r = s->at(ticket);
    if (r.ticket != ticket || r.state == ReqState::Free) return set_error(HNSW_ERR_INVALID_ARGUMENT, "unknown ticket");
    *done = r.state == ReqState::Done ? 1 : 0;
    return HNSW_OK;
}

int hnsw_gpu_wait(hnsw_gpu_server* s, uint64_t ticket, uint32_t timeout_ms, uint64_t* keys, float* dist,
                  uint32_t* count, int32_t* status, double* latency_us) {
    if (!s || !count || !status) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    std::unique_lock<std::mutex> lock(s->mu);
    Request& r = s->at(ticket);
    if (r.ticket != ticket || r.state == ReqState::Free) return set_error(HNSW_ERR_INVALID_ARGUMENT, "unknown ticket");
    const auto deadline = Clock::now() + std::chrono::milliseconds(timeout_ms);
    while (r.state != ReqState::Done) {
        if (s->cv_done.wait_until(lock, deadline) == std::cv_status::timeout && r.state != ReqState::Done)
            return set_error(HNSW_ERR_TIMEOUT, "request not finished before the timeout");
    }
    const uint64_t row = ticket % s->cap;
    *count = r.count;
    *status = r.status;
    if (keys) std::memcpy(keys, &s->keys[row * s->cfg.max_k], size_t(r.count) * 8);
    if (dist) std::memcpy(dist, &s->dist[row * s->cfg.max_k], size_t(r.count) * 4);
    if (latency_us) *latency_us = r.t_done - r.t_arrival;
    r.state = ReqState::Free;
    return HNSW_OK;
}

int hnsw_gpu_server_replay(hnsw_gpu_server* s, const float* queries, size_t n, const double* arrival_us,
                           const uint32_t* ks, const uint32_t* efs, const int32_t* filter_ids, uint64_t* out_keys,
                           float* out_dist, uint32_t* out_count, int32_t* out_status, double* out_latency_us) {
    if (!s || (n && (!queries || !arrival_us || !ks || !efs || !out_count || !out_status || !out_latency_us)))
        return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    const uint32_t dim = s->dim, K = s->cfg.max_k;
    std::vector<uint64_t> tickets(n, 0);
    std::vector<uint8_t> admitted(n, 0);
    std::atomic<size_t> submitted{0};
    const double t0 = now_us();
    // Feeder: admits each request at its arrival time (open loop).
    std::thread feeder([&] {
        size_t i = 0;
        while (i < n) {
            const double now = now_us() - t0;
            if (arrival_us[i] > now) {
                const double wait = arrival_us[i] - now;
                if (wait > 200) std::this_thread::sleep_for(std::chrono::microseconds(int64_t(wait - 100)));
                continue;
            }
            {
                std::lock_guard<std::mutex> g(s->mu);
                while (i < n && arrival_us[i] <= now_us() - t0) {
                    const int32_t fid = filter_ids ? filter_ids[i] : -1;
                    uint64_t t = 0;
                    if (submit_locked(s, queries + i * dim, ks[i], efs[i], fid, t0 + arrival_us[i], &t) == HNSW_OK) {
                        tickets[i] = t;
                        admitted[i] = 1;
                    }
                    ++i;
                }
            }
            submitted.store(i);
            s->cv_work.notify_one();
        }
    });
    // Collector: waits for each admitted request in order.
    for (size_t i = 0; i < n; ++i) {
        while (submitted.load() <= i) std::this_thread::sleep_for(std::chrono::microseconds(20));
        if (!admitted[i]) {
            out_count[i] = 0;
            out_status[i] = HNSW_ERR_ADMISSION_REJECTED;
            out_latency_us[i] = -1.0;
            continue;
        }
        int r = hnsw_gpu_wait(s, tickets[i], 60000, out_keys ? out_keys + i * K : nullptr,
                              out_dist ? out_dist + i * K : nullptr, &out_count[i], &out_status[i], &out_latency_us[i]);
        if (r != HNSW_OK) {
            out_status[i] = r;
            out_latency_us[i] = -1.0;
        }
    }
    feeder.join();
    return s->error;
}

int hnsw_gpu_server_stats(const hnsw_gpu_server* s, uint64_t* batches, uint64_t* queries) {
    if (!s) return set_error(HNSW_ERR_INVALID_ARGUMENT, "null argument");
    if (batches) *batches = s->launched_batches;
    if (queries) *queries = s->launched_queries;
    return HNSW_OK;
}

}  // extern "C"
