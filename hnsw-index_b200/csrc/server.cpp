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

// Resident mode: the request ring in mapped host memory, the serving
// kernel's device words and per-warp staging rows, and its scratch slot.
struct ResidentRing {
    uint32_t cap = 0;                 // ring rows (= request table rows)
    float* h_q = nullptr;             // cap x dim
    uint32_t* h_k = nullptr;
    uint32_t* h_ef = nullptr;
    int32_t* h_fid = nullptr;
    uint64_t* h_tail = nullptr;       // requests published
    uint32_t* h_stop = nullptr;
    uint64_t* h_keys = nullptr;       // outputs, cap x max_k
    float* h_dist = nullptr;
    uint32_t* h_count = nullptr;
    int32_t* h_status = nullptr;
    DBuf words;                       // claim (8 B), tail (8 B), stop (4 B), served (4 B)
    DBuf wq, wk, wef, wfu, wfid;      // per-warp staging rows
    Slot* slot = nullptr;             // spill areas and cold-list pool of the serving warps
    cudaEvent_t done = nullptr;
    bool running = false;
    uint32_t warps = 0;
    SearchGeometry geo;
    uint64_t published = 0;
    std::vector<uint64_t> ticket_of;  // ticket held by each ring row
    std::deque<uint64_t> inflight;    // ring positions published and not completed
    uint64_t launches = 0;
};

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
    ResidentRing ring;

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
    r.status = status;
    r.count = status == 0 ? std::min(b.h_count[i], r.k) : 0;
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

// Launches the serving kernel over the ring (caller holds mu).
int launch_resident(hnsw_gpu_server* s) {
    ResidentRing& R = s->ring;
    hnsw_gpu_index* gi = s->index;
    Slot* sl = R.slot;
    cudaStream_t st = sl->stream;
    const uint32_t n = gi->view.n;
    const uint32_t words = ((n + 31) / 32 + 3) & ~3u;
    const uint32_t tab_cap = (n + kColdChunk - 1) / kColdChunk + 2;
    const uint32_t chunks = uint32_t(sl->cold_pool.bytes / (size_t(kColdChunk) * 8));
    CU(sl->work.ensure(32), "cudaMalloc work counters");
    CU(cudaMemsetAsync(sl->work.p, 0, 32, st), "memset work counters");
    // A stop word raised to make the previous launch yield is lowered again.
    *reinterpret_cast<volatile uint32_t*>(R.h_stop) = 0;
    CU(cudaMemsetAsync(static_cast<unsigned char*>(R.words.p) + 16, 0, 4, st), "clear serving stop word");
    SearchArgs a;
    a.ix = gi->view;
    a.queries = R.wq.as<float>();
    a.nq = R.cap;
    a.k = s->cfg.max_k;
    a.ef = s->cfg.max_ef;
    a.ks = R.wk.as<uint32_t>();
    a.efs = R.wef.as<uint32_t>();
    a.quantized = s->cfg.quantized;
    if (s->words && s->cfg.filter_count) {
        a.filter_bits = s->bank.as<uint64_t>();
        a.filter_nbits = s->cfg.filter_nbits;
        a.filter_stride = s->words;
        a.filter_used = R.wfu.as<uint8_t>();
        a.filter_ids = R.wfid.as<uint32_t>();
        a.filter_by_node = s->cfg.filter_by_node;
    }
    uint64_t* dk = nullptr;
    float* dd = nullptr;
    uint32_t* dc = nullptr;
    int32_t* ds = nullptr;
    CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&dk), R.h_keys, 0), "mapped keys");
    CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&dd), R.h_dist, 0), "mapped dist");
    CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&dc), R.h_count, 0), "mapped counts");
    CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&ds), R.h_status, 0), "mapped statuses");
    a.out_keys = dk;
    a.out_dist = dd;
    a.out_count = dc;
    a.out_status = ds;
    a.out_stride = s->cfg.max_k;
    a.publish = 1;
    a.persistent = 1;
    a.spill_bits = sl->spill_bits.as<uint32_t>();
    a.spill_words = words;
    a.spill_slots = R.warps;
    a.cold_pool = sl->cold_pool.as<uint64_t>();
    a.cold_chunks = chunks;
    a.cold_next = sl->work.as<uint32_t>() + 2;
    a.cold_tab = sl->cold_tab.as<uint32_t>();
    a.cold_tab_cap = tab_cap;
    a.cold_slots = R.warps;
    ServeArgs sv;
    uint64_t* hw_tail = nullptr;
    uint32_t* hw_stop = nullptr;
    CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&hw_tail), R.h_tail, 0), "mapped tail");
    CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&hw_stop), R.h_stop, 0), "mapped stop");
    sv.host_tail = hw_tail;
    sv.host_stop = hw_stop;
    unsigned char* w = static_cast<unsigned char*>(R.words.p);
    sv.claim = reinterpret_cast<unsigned long long*>(w);
    sv.tail = reinterpret_cast<volatile uint64_t*>(w + 8);
    sv.stop = reinterpret_cast<volatile uint32_t*>(w + 16);
    sv.served = reinterpret_cast<uint32_t*>(w + 20);
    float* rq = nullptr;
    uint32_t *rk = nullptr, *ref = nullptr;
    int32_t* rfid = nullptr;
    CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&rq), R.h_q, 0), "mapped ring queries");
    CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&rk), R.h_k, 0), "mapped ring k");
    CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&ref), R.h_ef, 0), "mapped ring ef");
    CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&rfid), R.h_fid, 0), "mapped ring filters");
    sv.rq = rq;
    sv.rk = rk;
    sv.ref = ref;
    sv.rfid = rfid;
    sv.ring_cap = R.cap;
    sv.wq = R.wq.as<float>();
    sv.wk = R.wk.as<uint32_t>();
    sv.wef = R.wef.as<uint32_t>();
    sv.wfu = R.wfu.as<uint8_t>();
    sv.wfid = R.wfid.as<uint32_t>();
    int clock_khz = 0;
    if (cudaDeviceGetAttribute(&clock_khz, cudaDevAttrClockRate, gi->device) != cudaSuccess || clock_khz <= 0)
        clock_khz = 1965000;
    sv.idle_budget = (long long)s->cfg.idle_us * (clock_khz / 1000);
    sv.filter_rows = s->cfg.filter_count;
    sv.err = reinterpret_cast<uint32_t*>(w + 24);
    uint32_t launched = 0;
    CU(launch_serve(a, R.geo, sv, gi->num_sms, st, &launched), "serving kernel");
    CU(cudaEventRecord(R.done, st), "record serving event");
    R.running = true;
    ++R.launches;
    ++s->launched_batches;
    return HNSW_OK;
}

// Resident mode, one pass (the caller holds mu): harvest the ring rows whose
// status is out (overflowed queries go to `retry` for the batch path),
// publish pending requests into free rows, and launch the serving kernel
// when it is not running and requests wait. Returns whether anything moved.
bool resident_step(hnsw_gpu_server* s, std::vector<uint64_t>& retry, bool retry_busy) {
    ResidentRing& R = s->ring;
    const uint32_t K = s->cfg.max_k;
    bool any = false;
    const double t = now_us();
    for (auto it = R.inflight.begin(); it != R.inflight.end();) {
        const uint32_t row = uint32_t(*it % R.cap);
        const int32_t st = reinterpret_cast<volatile int32_t*>(R.h_status)[row];
        if (st == kUnpublished) {
            ++it;
            continue;
        }
        std::atomic_thread_fence(std::memory_order_acquire);
        const uint64_t ticket = R.ticket_of[row];
        if (st == kRetrying) {
            retry.push_back(ticket);
        } else {
            Request& r = s->at(ticket);
            const uint64_t rrow = ticket % s->cap;
            r.status = st;
            r.count = st == 0 ? std::min(R.h_count[row], r.k) : 0;
            std::memcpy(&s->keys[rrow * K], R.h_keys + size_t(row) * K, size_t(r.count) * 8);
            std::memcpy(&s->dist[rrow * K], R.h_dist + size_t(row) * K, size_t(r.count) * 4);
            r.t_done = t;
            r.state = ReqState::Done;
        }
        it = R.inflight.erase(it);
        any = true;
    }
    // Ring position p uses row p % cap, so a position is published only when
    // the oldest unharvested one is less than cap positions behind it (rows
    // finish out of order; a count of inflight rows would not say which).
    bool published = false;
    while (!s->pending.empty() && (R.inflight.empty() || R.published - R.inflight.front() < R.cap)) {
        const uint64_t ticket = s->pending.front();
        s->pending.pop_front();
        Request& r = s->at(ticket);
        r.state = ReqState::Inflight;
        const uint64_t pos = R.published++;
        const uint32_t row = uint32_t(pos % R.cap);
        R.ticket_of[row] = ticket;
        std::memcpy(R.h_q + size_t(row) * s->dim, &s->q[(ticket % s->cap) * s->dim], size_t(s->dim) * 4);
        R.h_k[row] = r.k;
        R.h_ef[row] = r.ef;
        R.h_fid[row] = r.filter_id;
        reinterpret_cast<volatile int32_t*>(R.h_status)[row] = kUnpublished;
        R.inflight.push_back(pos);
        ++s->launched_queries;
        published = true;
    }
    if (published) {
        std::atomic_thread_fence(std::memory_order_release);
        *reinterpret_cast<volatile uint64_t*>(R.h_tail) = R.published;
        any = true;
    }
    if (R.running && cudaEventQuery(R.done) != cudaErrorNotReady) {
        R.running = false;
        // A request the kernel refused (its own checks of the ring row).
        uint32_t err[2] = {0, 0};
        if (cudaMemcpy(err, static_cast<unsigned char*>(R.words.p) + 24, 8, cudaMemcpyDeviceToHost) != cudaSuccess)
            s->error = HNSW_ERR_CUDA;
        else if (err[0] && s->error == HNSW_OK)
            s->error = HNSW_ERR_INVALID_ARGUMENT;
    }
    const bool retrying = !retry.empty() || retry_busy;
    if (R.running && retrying) {
        // Overflowed queries need the retry kernels, which need SMs the
        // serving kernel holds: ask it to leave after its current requests,
        // and launch it again once the retry batch is done.
        *reinterpret_cast<volatile uint32_t*>(R.h_stop) = 1;
    }
    if (!R.running && !R.inflight.empty() && !retrying) {
        const int e = launch_resident(s);
        if (e != HNSW_OK) s->error = e;
    }
    return any;
}

void dispatch_loop(hnsw_gpu_server* s) {
    DeviceGuard dg(s->index->device);
    std::vector<uint64_t> take;
    std::vector<uint64_t> retry;
    double stop_deadline = 0.0;
    while (true) {
        std::unique_lock<std::mutex> lock(s->mu);
        if (s->cfg.resident) {
            // Serving kernel first; overflowed queries wait for the batch slot.
            bool busy_batch = false;
            for (BatchSlot& b : s->batches) {
                if (!b.busy) continue;
                if (cudaEventQuery(b.done) == cudaSuccess) harvest(s, b, true);
                else busy_batch = true;
            }
            bool any = resident_step(s, retry, busy_batch);
            if (!retry.empty() && !busy_batch) {
                BatchSlot& b = s->batches[0];
                b.busy = true;
                const size_t nb = std::min<size_t>(retry.size(), s->cfg.max_batch);
                b.tickets.assign(retry.begin(), retry.begin() + nb);
                retry.erase(retry.begin(), retry.begin() + nb);
                const int r = stage_and_launch(s, b, b.tickets);
                if (r != HNSW_OK) {
                    s->error = r;
                    for (uint64_t t : b.tickets) {
                        Request& q = s->at(t);
                        q.status = r;
                        q.count = 0;
                        q.t_done = now_us();
                        q.state = ReqState::Done;
                    }
                    b.busy = false;
                    b.tickets.clear();
                }
                any = true;
            }
            if (any) s->cv_done.notify_all();
            if (s->stop && s->pending.empty() && s->ring.inflight.empty() && retry.empty() && !busy_batch) break;
            if (s->stop) {
                // Stopping: requests get idle_us plus 10 s to finish; any left
                // then (a kernel that cannot make progress) end with TIMEOUT so
                // that stopping always returns.
                if (stop_deadline == 0.0) stop_deadline = now_us() + 1e7 + double(s->cfg.idle_us);
                if (now_us() > stop_deadline && !busy_batch) {
                    const double t = now_us();
                    auto fail = [&](uint64_t ticket) {
                        Request& q = s->at(ticket);
                        q.status = HNSW_ERR_TIMEOUT;
                        q.count = 0;
                        q.t_done = t;
                        q.state = ReqState::Done;
                    };
                    for (uint64_t pos : s->ring.inflight) fail(s->ring.ticket_of[pos % s->ring.cap]);
                    for (uint64_t ticket : s->pending) fail(ticket);
                    for (uint64_t ticket : retry) fail(ticket);
                    s->ring.inflight.clear();
                    s->pending.clear();
                    retry.clear();
                    s->error = HNSW_ERR_TIMEOUT;
                    s->cv_done.notify_all();
                    break;
                }
            }
            if (!any) {
                if (s->ring.inflight.empty() && s->pending.empty() && !busy_batch && retry.empty()) {
                    s->cv_work.wait_for(lock, std::chrono::milliseconds(2));
                } else {
                    lock.unlock();
                    std::this_thread::sleep_for(std::chrono::microseconds(5));
                }
            }
            continue;
        }
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
    c->resident = 0;
    c->idle_us = 20000;
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
    if (cfg.resident) {
        ResidentRing& R = s->ring;
        if (!s->cfg.idle_us) s->cfg.idle_us = 20000;
        if (s->cap > (uint64_t(1) << 30)) return set_error(HNSW_ERR_INVALID_ARGUMENT, "ring too large");
        R.cap = uint32_t(s->cap);
        const size_t C = R.cap;
        CU(cudaHostAlloc(&R.h_q, C * s->dim * 4, cudaHostAllocMapped), "mapped ring queries");
        CU(cudaHostAlloc(&R.h_k, C * 4, cudaHostAllocMapped), "mapped ring k");
        CU(cudaHostAlloc(&R.h_ef, C * 4, cudaHostAllocMapped), "mapped ring ef");
        CU(cudaHostAlloc(&R.h_fid, C * 4, cudaHostAllocMapped), "mapped ring filters");
        CU(cudaHostAlloc(&R.h_tail, 64, cudaHostAllocMapped), "mapped ring tail");
        CU(cudaHostAlloc(&R.h_stop, 64, cudaHostAllocMapped), "mapped ring stop");
        CU(cudaHostAlloc(&R.h_keys, C * cfg.max_k * 8, cudaHostAllocMapped), "mapped ring keys");
        CU(cudaHostAlloc(&R.h_dist, C * cfg.max_k * 4, cudaHostAllocMapped), "mapped ring dist");
        CU(cudaHostAlloc(&R.h_count, C * 4, cudaHostAllocMapped), "mapped ring counts");
        CU(cudaHostAlloc(&R.h_status, C * 4, cudaHostAllocMapped), "mapped ring statuses");
        *reinterpret_cast<volatile uint64_t*>(R.h_tail) = 0;
        *reinterpret_cast<volatile uint32_t*>(R.h_stop) = 0;
        for (size_t i = 0; i < C; ++i) {
            R.h_status[i] = kUnpublished;
            R.h_k[i] = 0;
            R.h_ef[i] = 0;
            R.h_fid[i] = -1;
        }
        std::memset(R.h_q, 0, C * s->dim * 4);
        R.ticket_of.assign(C, 0);
        const uint32_t ef_max = std::max(cfg.max_ef, cfg.max_k);
        R.geo = pick_geometry(ef_max, index->view.dp, index->view.dc, true, cfg.filter_count > 0);
        R.geo.stage_rows = 0;
        CU(serve_warps(R.geo, index->view.dp, index->view.dc, index->num_sms, &R.warps), "serving occupancy");
        int r = index->slots.acquire(&R.slot);
        if (r != HNSW_OK) return r;
        Slot* sl = R.slot;
        const uint32_t n = index->view.n;
        const uint32_t words = ((n + 31) / 32 + 3) & ~3u;
        const uint32_t tab_cap = (n + kColdChunk - 1) / kColdChunk + 2;
        const uint64_t want = std::max<uint64_t>((uint64_t(n) * 8 + kColdChunk - 1) / kColdChunk, uint64_t(R.warps) * 32);
        const uint32_t chunks = uint32_t(std::min<uint64_t>(want, 1u << 18));
        CU(sl->spill_bits.ensure(size_t(R.warps) * words * 4), "cudaMalloc serving spill bitmaps");
        CU(cudaMemset(sl->spill_bits.p, 0, sl->spill_bits.bytes), "memset serving spill bitmaps");
        CU(sl->cold_pool.ensure(size_t(chunks) * kColdChunk * 8), "cudaMalloc serving cold pool");
        CU(sl->cold_tab.ensure(size_t(R.warps) * tab_cap * 4), "cudaMalloc serving chunk tables");
        CU(R.words.ensure(32), "cudaMalloc serving words");
        CU(cudaMemset(R.words.p, 0, 32), "memset serving words");
        CU(R.wq.ensure(size_t(R.warps) * s->dim * 4), "cudaMalloc staging queries");
        CU(R.wk.ensure(size_t(R.warps) * 4), "cudaMalloc staging k");
        CU(R.wef.ensure(size_t(R.warps) * 4), "cudaMalloc staging ef");
        CU(R.wfu.ensure(size_t(R.warps)), "cudaMalloc staging filter flags");
        CU(R.wfid.ensure(size_t(R.warps) * 4), "cudaMalloc staging filter ids");
        CU(cudaEventCreateWithFlags(&R.done, cudaEventDisableTiming), "serving event");
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
    ResidentRing& R = s->ring;
    if (R.h_stop) {
        // The kernel leaves at the stop word, or after its idle budget.
        *reinterpret_cast<volatile uint32_t*>(R.h_stop) = 1;
        std::atomic_thread_fence(std::memory_order_seq_cst);
        if (R.done) cudaEventSynchronize(R.done);
    }
    if (R.done) cudaEventDestroy(R.done);
    for (void* p : {(void*)R.h_q, (void*)R.h_k, (void*)R.h_ef, (void*)R.h_fid, (void*)R.h_tail, (void*)R.h_stop,
                    (void*)R.h_keys, (void*)R.h_dist, (void*)R.h_count, (void*)R.h_status})
        if (p) cudaFreeHost(p);
    for (DBuf* b : {&R.words, &R.wq, &R.wk, &R.wef, &R.wfu, &R.wfid}) b->release();
    if (R.slot) s->index->slots.release(R.slot);
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
