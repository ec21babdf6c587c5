// CPU ORACLE — test infrastructure, not product code.
//
// A plain C++ restatement of the hnsw-index crate's query path, used only by
// tests/, __graft_entry__.smoke() and the CPU-baseline / reference legs of
// bench.py, as the checker the CUDA path is compared against. Nothing in the
// product library links or calls this file.
//
// Every function names the reference file:line it restates (paths are within
// the hnsw-index crate). Pinned by the reference's own known answers (see
// tests/test_oracle_golden.py): SplitMix64 outputs, the golden components of
// the synthetic generator (tests/recall.rs:130-138), CRC-32 check values, scalar kernel known answers, metric known
// answers (IP -0.0), brute-force tie breaking, the complete-graph exactness
// case and the recall pins.
//
// Compile with -ffp-contract=off: the reference (Rust) never contracts a*b+c,
// and every FMA below is explicit.

#include <immintrin.h>
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <queue>
#include <thread>
#include <vector>

namespace {

// ---------------------------------------------------------------------------
// f32 kernels in the AVX2 backend's summation order
// (src/kernels/x86.rs:32-131): four FMA chains of eight lanes over 32-float
// steps, an 8-wide tail into chain 0, lane-wise (c0+c1)+(c2+c3), the
// horizontal sum ((l0+l4)+(l1+l5))+((l2+l6)+(l3+l7)) (x86.rs:19-26), then a
// scalar tail without FMA.
// ---------------------------------------------------------------------------

inline float hsum8(const float* v) {
    return ((v[0] + v[4]) + (v[1] + v[5])) + ((v[2] + v[6]) + (v[3] + v[7]));
}

// Portable restatement (fmaf per lane is exactly what _mm256_fmadd_ps does).
float dot_avx2order_portable(const float* a, const float* b, size_t len) {
    float acc[4][8] = {};
    size_t i = 0;
    for (; i + 32 <= len; i += 32)
        for (int c = 0; c < 4; ++c)
            for (int l = 0; l < 8; ++l)
                acc[c][l] = std::fmaf(a[i + 8 * c + l], b[i + 8 * c + l], acc[c][l]);
    for (; i + 8 <= len; i += 8)
        for (int l = 0; l < 8; ++l) acc[0][l] = std::fmaf(a[i + l], b[i + l], acc[0][l]);
    float v[8];
    for (int l = 0; l < 8; ++l) v[l] = (acc[0][l] + acc[1][l]) + (acc[2][l] + acc[3][l]);
    float sum = hsum8(v);
    for (; i < len; ++i) sum += a[i] * b[i];
    return sum;
}

float l2_avx2order_portable(const float* a, const float* b, size_t len) {
    float acc[4][8] = {};
    size_t i = 0;
    for (; i + 32 <= len; i += 32)
        for (int c = 0; c < 4; ++c)
            for (int l = 0; l < 8; ++l) {
                float d = a[i + 8 * c + l] - b[i + 8 * c + l];
                acc[c][l] = std::fmaf(d, d, acc[c][l]);
            }
    for (; i + 8 <= len; i += 8)
        for (int l = 0; l < 8; ++l) {
            float d = a[i + l] - b[i + l];
            acc[0][l] = std::fmaf(d, d, acc[0][l]);
        }
    float v[8];
    for (int l = 0; l < 8; ++l) v[l] = (acc[0][l] + acc[1][l]) + (acc[2][l] + acc[3][l]);
    float sum = hsum8(v);
    for (; i < len; ++i) {
        float d = a[i] - b[i];
        sum += d * d;
    }
    return sum;
}

// Intrinsics version (same bits; used when the CPU has AVX2+FMA).
__attribute__((target("avx2,fma"))) float dot_avx2(const float* a, const float* b, size_t len) {
    __m256 acc0 = _mm256_setzero_ps(), acc1 = _mm256_setzero_ps();
    __m256 acc2 = _mm256_setzero_ps(), acc3 = _mm256_setzero_ps();
    size_t i = 0;
    for (; i + 32 <= len; i += 32) {
        acc0 = _mm256_fmadd_ps(_mm256_loadu_ps(a + i), _mm256_loadu_ps(b + i), acc0);
        acc1 = _mm256_fmadd_ps(_mm256_loadu_ps(a + i + 8), _mm256_loadu_ps(b + i + 8), acc1);
        acc2 = _mm256_fmadd_ps(_mm256_loadu_ps(a + i + 16), _mm256_loadu_ps(b + i + 16), acc2);
        acc3 = _mm256_fmadd_ps(_mm256_loadu_ps(a + i + 24), _mm256_loadu_ps(b + i + 24), acc3);
    }
    for (; i + 8 <= len; i += 8)
        acc0 = _mm256_fmadd_ps(_mm256_loadu_ps(a + i), _mm256_loadu_ps(b + i), acc0);
    float v[8];
    _mm256_storeu_ps(v, _mm256_add_ps(_mm256_add_ps(acc0, acc1), _mm256_add_ps(acc2, acc3)));
    float sum = hsum8(v);
    for (; i < len; ++i) sum += a[i] * b[i];
    return sum;
}

__attribute__((target("avx2,fma"))) float l2_avx2(const float* a, const float* b, size_t len) {
    __m256 acc0 = _mm256_setzero_ps(), acc1 = _mm256_setzero_ps();
    __m256 acc2 = _mm256_setzero_ps(), acc3 = _mm256_setzero_ps();
    size_t i = 0;
    for (; i + 32 <= len; i += 32) {
        __m256 d0 = _mm256_sub_ps(_mm256_loadu_ps(a + i), _mm256_loadu_ps(b + i));
        __m256 d1 = _mm256_sub_ps(_mm256_loadu_ps(a + i + 8), _mm256_loadu_ps(b + i + 8));
        __m256 d2 = _mm256_sub_ps(_mm256_loadu_ps(a + i + 16), _mm256_loadu_ps(b + i + 16));
        __m256 d3 = _mm256_sub_ps(_mm256_loadu_ps(a + i + 24), _mm256_loadu_ps(b + i + 24));
        acc0 = _mm256_fmadd_ps(d0, d0, acc0);
        acc1 = _mm256_fmadd_ps(d1, d1, acc1);
        acc2 = _mm256_fmadd_ps(d2, d2, acc2);
        acc3 = _mm256_fmadd_ps(d3, d3, acc3);
    }
    for (; i + 8 <= len; i += 8) {
        __m256 d = _mm256_sub_ps(_mm256_loadu_ps(a + i), _mm256_loadu_ps(b + i));
        acc0 = _mm256_fmadd_ps(d, d, acc0);
    }
    float v[8];
    _mm256_storeu_ps(v, _mm256_add_ps(_mm256_add_ps(acc0, acc1), _mm256_add_ps(acc2, acc3)));
    float sum = hsum8(v);
    for (; i < len; ++i) {
        float d = a[i] - b[i];
        sum += d * d;
    }
    return sum;
}

bool have_avx2() {
    static const bool ok = __builtin_cpu_supports("avx2") && __builtin_cpu_supports("fma");
    return ok;
}

inline float k_dot(const float* a, const float* b, size_t n) {
    return have_avx2() ? dot_avx2(a, b, n) : dot_avx2order_portable(a, b, n);
}
inline float k_l2(const float* a, const float* b, size_t n) {
    return have_avx2() ? l2_avx2(a, b, n) : l2_avx2order_portable(a, b, n);
}

// Scalar backend: one accumulator, strict left to right (src/kernels/scalar.rs:7-22).
float dot_scalar(const float* a, const float* b, size_t n) {
    float s = 0.0f;
    for (size_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}
float l2_scalar(const float* a, const float* b, size_t n) {
    float s = 0.0f;
    for (size_t i = 0; i < n; ++i) {
        float d = a[i] - b[i];
        s += d * d;
    }
    return s;
}

enum Metric : uint8_t { L2 = 0, IP = 1, COS = 2 };

// Metric::distance (src/metric.rs:35-41).
inline float metric_distance(int metric, const float* a, const float* b, size_t n) {
    switch (metric) {
        case L2: return k_l2(a, b, n);
        case IP: return -k_dot(a, b, n);
        default: return 1.0f - k_dot(a, b, n);
    }
}

// int8 kernels: exact integer sums (src/kernels/int8.rs:13-48).
int64_t i8_dot(const int8_t* a, const int8_t* b, size_t n) {
    int64_t s = 0;
    for (size_t i = 0; i < n; ++i) s += int64_t(a[i]) * int64_t(b[i]);
    return s;
}
int64_t i8_l2(const int8_t* a, const int8_t* b, size_t n) {
    int64_t s = 0;
    for (size_t i = 0; i < n; ++i) {
        int64_t d = int64_t(a[i]) - int64_t(b[i]);
        s += d * d;
    }
    return s;
}

// ScalarQuantizer::encode_into (src/quantization.rs:73-81): inv = 1/scale in
// f32, code = clamp(round_half_away((x - o) * inv), -127, 127).
void sq_encode(const float* x, const float* offset, float scale, size_t dim, int8_t* out) {
    float inv = 1.0f / scale;
    for (size_t i = 0; i < dim; ++i) {
        float v = std::round((x[i] - offset[i]) * inv);
        v = std::min(127.0f, std::max(-127.0f, v));
        out[i] = int8_t(v);
    }
}

// ScalarQuantizer::distance (src/quantization.rs:85-92).
inline float sq_distance(int metric, float scale, const int8_t* a, const int8_t* b, size_t n) {
    float s2 = scale * scale;
    switch (metric) {
        case L2: return float(i8_l2(a, b, n)) * s2;
        case IP: return -float(i8_dot(a, b, n)) * s2;
        default: return 1.0f - float(i8_dot(a, b, n)) * s2;
    }
}

// total_cmp of f32 (Rust core::f32::total_cmp).
inline int32_t total_key(float f) {
    int32_t b;
    std::memcpy(&b, &f, 4);
    b ^= int32_t(uint32_t(b >> 31) >> 1);
    return b;
}

// Candidate ordering: (total_cmp distance, id) (src/hnsw/search.rs:36-44).
struct Cand {
    float d;
    uint32_t id;
};
inline bool cand_less(const Cand& a, const Cand& b) {
    int32_t ka = total_key(a.d), kb = total_key(b.d);
    return ka != kb ? ka < kb : a.id < b.id;
}
struct CandLess {
    bool operator()(const Cand& a, const Cand& b) const { return cand_less(a, b); }
};
struct CandGreater {
    bool operator()(const Cand& a, const Cand& b) const { return cand_less(b, a); }
};

// ---------------------------------------------------------------------------
// SplitMix64 + Box-Muller + Lemire (src/synthetic.rs:23-60).
// ---------------------------------------------------------------------------
inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
struct SplitMix64 {
    uint64_t s;
    uint64_t next() {
        s += 0x9E3779B97F4A7C15ULL;
        return mix64(s);
    }
    double next_f64() { return double(next() >> 11) * (1.0 / double(1ULL << 53)); }
    uint64_t below(uint64_t n) { return uint64_t((__uint128_t(next()) * n) >> 64); }
    double gaussian() {
        double u1 = 1.0 - next_f64();
        double u2 = next_f64();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

// ---------------------------------------------------------------------------
// A loaded index (format v1, src/hnsw/io.rs:3-28). The oracle trusts files
// that the validating loader of the product library has accepted; it checks
// only the envelope and lengths.
// ---------------------------------------------------------------------------
struct Index {
    int metric = 0;
    uint32_t dim = 0, m = 0, m0 = 0, n = 0, entry = 0xFFFFFFFFu;
    uint8_t top = 0;
    bool quantized = false;
    std::vector<uint64_t> keys;
    std::vector<uint8_t> levels, deleted;
    std::vector<float> vectors;
    // layer 0: (m0+1) words per node (count, ids)
    std::vector<uint32_t> l0;
    // upper layers: per node, level*(m+1) words
    std::vector<std::vector<uint32_t>> upper;
    std::vector<float> offset;
    float scale = 1.0f;
    std::vector<int8_t> codes;
    size_t live = 0;

    const float* vec(uint32_t id) const { return vectors.data() + size_t(id) * dim; }
    const uint32_t* list(uint32_t id, unsigned layer, uint32_t* count) const {
        if (layer == 0) {
            const uint32_t* b = l0.data() + size_t(id) * (m0 + 1);
            *count = std::min(b[0], m0);
            return b + 1;
        }
        const uint32_t* b = upper[id].data() + size_t(layer - 1) * (m + 1);
        *count = std::min(b[0], m);
        return b + 1;
    }
};

uint32_t crc_table[256];
bool crc_ready = false;
uint32_t crc32(const uint8_t* p, size_t n) {
    if (!crc_ready) {
        for (uint32_t i = 0; i < 256; ++i) {
            uint32_t c = i;
            for (int k = 0; k < 8; ++k) c = (c & 1) ? (c >> 1) ^ 0xEDB88320u : (c >> 1);
            crc_table[i] = c;
        }
        crc_ready = true;
    }
    uint32_t c = 0xFFFFFFFFu;
    for (size_t i = 0; i < n; ++i) c = (c >> 8) ^ crc_table[(c ^ p[i]) & 0xFF];
    return ~c;
}

struct Rd {
    const uint8_t* p;
    size_t n, pos;
    bool ok = true;
    const uint8_t* take(size_t k) {
        if (!ok || k > n - pos) {
            ok = false;
            return nullptr;
        }
        const uint8_t* r = p + pos;
        pos += k;
        return r;
    }
    template <class T>
    T get() {
        T v{};
        const uint8_t* b = take(sizeof(T));
        if (b) std::memcpy(&v, b, sizeof(T));
        return v;
    }
};

// ---------------------------------------------------------------------------
// Search (src/hnsw/search.rs:49-161, src/hnsw/mod.rs:460-511).
// ---------------------------------------------------------------------------
struct Stats {
    uint64_t dist0 = 0, exp0 = 0, dist_up = 0, exp_up = 0;
};

struct Scratch {
    std::vector<uint16_t> marks;
    uint16_t epoch = 0;
    void reset(size_t n) {  // VisitedSet::reset (src/hnsw/scratch.rs:25-33)
        if (marks.size() < n) marks.resize(n, 0);
        epoch = uint16_t(epoch + 1);
        if (epoch == 0) {
            std::fill(marks.begin(), marks.end(), 0);
            epoch = 1;
        }
    }
    bool insert(uint32_t id) {
        if (marks[id] == epoch) return false;
        marks[id] = epoch;
        return true;
    }
};

struct Filter {
    // Key bitmap: key admitted iff key < nbits and bit set. nullptr = no filter.
    // With by_node the bitmap is indexed by node id instead (the same closure
    // evaluated once per node, for indexes whose keys are sparse u64 values).
    const uint64_t* bits = nullptr;
    uint64_t nbits = 0;
    bool by_node = false;
    bool accept(uint64_t key) const {
        if (!bits) return true;
        return key < nbits && ((bits[key >> 6] >> (key & 63)) & 1);
    }
};

template <class Dist, class Admit>
Cand greedy_closest(const Index& ix, Cand start, unsigned layer, const Dist& dist, Stats& st) {
    Cand best = start;
    for (;;) {
        uint32_t from = best.id, cnt;
        const uint32_t* ids = ix.list(from, layer, &cnt);
        st.exp_up++;
        for (uint32_t j = 0; j < cnt; ++j) {
            float d = dist(ids[j]);
            st.dist_up++;
            if (d < best.d) best = Cand{d, ids[j]};
        }
        if (best.id == from) return best;
    }
}

template <class Dist, class Admit>
std::vector<Cand> search_layer0(const Index& ix, Scratch& sc, Cand ep, size_t ef, const Dist& dist,
                                const Admit& admit, Stats& st) {
    sc.reset(ix.n);
    std::priority_queue<Cand, std::vector<Cand>, CandGreater> cands;  // min-heap
    std::priority_queue<Cand, std::vector<Cand>, CandLess> results;   // max-heap
    if (sc.insert(ep.id)) {
        cands.push(ep);
        if (admit(ep.id)) {
            results.push(ep);
            if (results.size() > ef) results.pop();
        }
    }
    while (!cands.empty()) {
        Cand cur = cands.top();
        cands.pop();
        if (results.size() >= ef && !results.empty() && cur.d > results.top().d) break;
        uint32_t cnt;
        const uint32_t* ids = ix.list(cur.id, 0, &cnt);
        st.exp0++;
        for (uint32_t j = 0; j < cnt; ++j) {
            uint32_t nb = ids[j];
            if (!sc.insert(nb)) continue;
            float d = dist(nb);
            st.dist0++;
            bool improves = results.size() < ef || (!results.empty() && d < results.top().d);
            if (improves) {
                Cand c{d, nb};
                cands.push(c);
                if (admit(nb)) {
                    results.push(c);
                    if (results.size() > ef) results.pop();
                }
            }
        }
    }
    std::vector<Cand> out;
    out.reserve(results.size());
    while (!results.empty()) {
        out.push_back(results.top());
        results.pop();
    }
    std::sort(out.begin(), out.end(), CandLess());
    return out;
}

enum Status : int32_t {
    OK = 0,
    DIMENSION_MISMATCH = 1,
    NON_FINITE_VECTOR = 3,
    ZERO_VECTOR = 4,
    QUANTIZATION_DISABLED = 7,
};

// check + normalized + prepare_query (src/vector.rs:22-45,90-104).
int32_t prepare_query(int metric, const float* q, size_t dim, float* out) {
    double norm = 0.0;
    for (size_t i = 0; i < dim; ++i) {
        if (!std::isfinite(q[i])) return NON_FINITE_VECTOR;
        norm += double(q[i]) * double(q[i]);
    }
    if (norm > double(3.40282346638528859812e+38F) / 8.0) return NON_FINITE_VECTOR;
    if (metric == COS) {
        if (norm == 0.0) return ZERO_VECTOR;
        double inv = 1.0 / std::sqrt(norm);
        for (size_t i = 0; i < dim; ++i) out[i] = float(double(q[i]) * inv);
    } else {
        std::memcpy(out, q, dim * 4);
    }
    return OK;
}

struct Hit {
    uint64_t key;
    float d;
};
inline bool hit_less(const Hit& a, const Hit& b) {  // Neighbor::cmp_by_distance (src/neighbor.rs:17-21)
    int32_t ka = total_key(a.d), kb = total_key(b.d);
    return ka != kb ? ka < kb : a.key < b.key;
}

// HnswIndex::search_impl (src/hnsw/mod.rs:460-511), one query.
int32_t search_one(const Index& ix, Scratch& sc, const float* query, size_t k, size_t ef, bool quantized,
                   const Filter& filter, std::vector<Hit>& out, Stats& st) {
    out.clear();
    std::vector<float> q(ix.dim);
    int32_t s = prepare_query(ix.metric, query, ix.dim, q.data());
    if (s != OK) return s;
    if (quantized && !ix.quantized) return QUANTIZATION_DISABLED;
    if (k == 0 || ix.live == 0) return OK;
    ef = std::max(ef, k);
    auto admit = [&](uint32_t id) {
        return !ix.deleted[id] && filter.accept(filter.by_node ? uint64_t(id) : ix.keys[id]);
    };
    auto exact = [&](uint32_t id) { return metric_distance(ix.metric, q.data(), ix.vec(id), ix.dim); };
    std::vector<Cand> found;
    if (ix.entry == 0xFFFFFFFFu) return OK;
    if (!quantized) {
        Cand ep{exact(ix.entry), ix.entry};
        st.dist_up++;
        for (int layer = ix.top; layer >= 1; --layer)
            ep = greedy_closest<decltype(exact), decltype(admit)>(ix, ep, unsigned(layer), exact, st);
        found = search_layer0(ix, sc, ep, ef, exact, admit, st);
    } else {
        std::vector<int8_t> code(ix.dim);
        sq_encode(q.data(), ix.offset.data(), ix.scale, ix.dim, code.data());
        auto approx = [&](uint32_t id) {
            return sq_distance(ix.metric, ix.scale, code.data(), ix.codes.data() + size_t(id) * ix.dim, ix.dim);
        };
        Cand ep{approx(ix.entry), ix.entry};
        st.dist_up++;
        for (int layer = ix.top; layer >= 1; --layer)
            ep = greedy_closest<decltype(approx), decltype(admit)>(ix, ep, unsigned(layer), approx, st);
        found = search_layer0(ix, sc, ep, ef, approx, admit, st);
        for (auto& c : found) c.d = exact(c.id);
    }
    out.reserve(found.size());
    for (auto& c : found) out.push_back(Hit{ix.keys[c.id], c.d});
    std::sort(out.begin(), out.end(), hit_less);
    if (out.size() > k) out.resize(k);
    return OK;
}

template <class F>
void parallel_for(size_t n, int threads, F&& f) {
    if (threads <= 0) threads = int(std::max(1u, std::thread::hardware_concurrency()));
    if (threads == 1 || n < 2) {
        for (size_t i = 0; i < n; ++i) f(0, i);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&, t] {
            for (;;) {
                size_t i = next.fetch_add(1, std::memory_order_relaxed);
                if (i >= n) break;
                f(t, i);
            }
        });
    for (auto& th : pool) th.join();
}


// ---------------------------------------------------------------------------
// Construction, restated for making index files on the reference side:
// HnswIndex::insert / insert_batch (src/hnsw/mod.rs:225-349), sample_level,
// link, install_own_neighbors, connect, write_shrunk, select_neighbors and
// extend_candidates (src/hnsw/build.rs:19-222), the fixed-capacity lists of
// src/hnsw/graph.rs:26-135 (count word, then ids; writers publish the ids
// before the count), and search_layer over any layer with several entry
// points (src/hnsw/search.rs:81-142). One thread links the nodes in id order,
// which is the sequence of `insert` calls; more threads link them
// concurrently as link_parallel does (mod.rs:336-346), each node behind its
// own lock, the entry point behind the promotion lock.
// ---------------------------------------------------------------------------
constexpr uint64_t kNoEntry = ~0ull;
constexpr unsigned kMaxLevel = 31;

uint8_t sample_level(uint64_t seed, uint32_t id, double ml) {  // build.rs:19-28
    const uint64_t h = mix64(seed ^ mix64(uint64_t(id) + 0x9E3779B97F4A7C15ULL));
    const double u = double((h >> 11) + 1) * (1.0 / double(1ULL << 53));
    const double level = std::floor(-std::log(u) * ml);
    return level >= double(kMaxLevel) ? uint8_t(kMaxLevel) : uint8_t(level);
}

struct Graph {
    size_t dim = 0;
    int metric = 0;
    uint32_t m = 0, m0 = 0, efc = 0;
    double ml = 0.0;
    int selection = 1;  // 0 simple, 1 heuristic
    bool extend = false, keep = false;
    uint64_t seed = 0;
    uint32_t n = 0;
    std::vector<float> vectors;
    std::vector<uint64_t> keys;
    std::vector<uint8_t> levels;
    std::vector<std::atomic<uint32_t>> l0;     // (m0 + 1) words per node
    std::vector<std::atomic<uint32_t>> upper;  // level * (m + 1) words per node
    std::vector<size_t> up_off;
    std::vector<std::mutex> locks;
    std::atomic<uint64_t> entry{kNoEntry};
    std::mutex promotion;

    const float* vec(uint32_t id) const { return vectors.data() + size_t(id) * dim; }
    float dist(const float* a, uint32_t b) const { return metric_distance(metric, a, vec(b), dim); }
    uint32_t capacity(unsigned layer) const { return layer == 0 ? m0 : m; }
    std::atomic<uint32_t>* block(uint32_t id, unsigned layer) {
        if (layer == 0) return l0.data() + size_t(id) * (m0 + 1);
        return upper.data() + up_off[id] + size_t(layer - 1) * (m + 1);
    }
    void read(uint32_t id, unsigned layer, std::vector<uint32_t>& out) {  // Links::read_into
        out.clear();
        std::atomic<uint32_t>* b = block(id, layer);
        const uint32_t c = std::min(b[0].load(std::memory_order_acquire), capacity(layer));
        for (uint32_t j = 0; j < c; ++j) out.push_back(b[1 + j].load(std::memory_order_relaxed));
    }
    void set(uint32_t id, unsigned layer, const std::vector<uint32_t>& ids) {  // Links::set
        std::atomic<uint32_t>* b = block(id, layer);
        for (size_t j = 0; j < ids.size(); ++j) b[1 + j].store(ids[j], std::memory_order_relaxed);
        b[0].store(uint32_t(ids.size()), std::memory_order_release);
    }
    bool try_push(uint32_t id, unsigned layer, uint32_t nb) {  // Links::try_push
        std::atomic<uint32_t>* b = block(id, layer);
        const uint32_t c = b[0].load(std::memory_order_relaxed);
        if (c >= capacity(layer)) return false;
        b[1 + c].store(nb, std::memory_order_relaxed);
        b[0].store(c + 1, std::memory_order_release);
        return true;
    }
};

struct BuildScratch {
    std::vector<uint16_t> marks;
    uint16_t epoch = 0;
    std::vector<uint32_t> ids;
    void reset(size_t n) {
        if (marks.size() < n) marks.resize(n, 0);
        epoch = uint16_t(epoch + 1);
        if (epoch == 0) {
            std::fill(marks.begin(), marks.end(), 0);
            epoch = 1;
        }
    }
    bool insert(uint32_t id) {
        if (marks[id] == epoch) return false;
        marks[id] = epoch;
        return true;
    }
};

// greedy_closest (search.rs:49-68) on the graph under construction.
Cand build_greedy(Graph& g, BuildScratch& sc, Cand best, unsigned layer, const float* q) {
    for (;;) {
        const uint32_t from = best.id;
        g.read(from, layer, sc.ids);
        for (uint32_t nb : sc.ids) {
            const float d = g.dist(q, nb);
            if (d < best.d) best = Cand{d, nb};
        }
        if (best.id == from) return best;
    }
}

// search_layer (search.rs:81-142) with the admission `n != self`.
std::vector<Cand> build_search_layer(Graph& g, BuildScratch& sc, const std::vector<Cand>& eps, size_t ef,
                                     unsigned layer, const float* q, uint32_t self) {
    sc.reset(g.n);
    std::priority_queue<Cand, std::vector<Cand>, CandGreater> cands;
    std::priority_queue<Cand, std::vector<Cand>, CandLess> results;
    for (const Cand& ep : eps) {
        if (!sc.insert(ep.id)) continue;
        cands.push(ep);
        if (ep.id != self) {
            results.push(ep);
            if (results.size() > ef) results.pop();
        }
    }
    std::vector<uint32_t> list;
    while (!cands.empty()) {
        const Cand cur = cands.top();
        cands.pop();
        if (results.size() >= ef && !results.empty() && cur.d > results.top().d) break;
        g.read(cur.id, layer, list);
        for (uint32_t nb : list) {
            if (!sc.insert(nb)) continue;
            const float d = g.dist(q, nb);
            const bool improves = results.size() < ef || (!results.empty() && d < results.top().d);
            if (!improves) continue;
            cands.push(Cand{d, nb});
            if (nb != self) {
                results.push(Cand{d, nb});
                if (results.size() > ef) results.pop();
            }
        }
    }
    std::vector<Cand> out;
    out.reserve(results.size());
    while (!results.empty()) {
        out.push_back(results.top());
        results.pop();
    }
    std::sort(out.begin(), out.end(), CandLess());
    return out;
}

// extend_candidates (build.rs:198-220).
std::vector<Cand> extend_candidates(Graph& g, uint32_t base_id, const float* base, const std::vector<Cand>& cands,
                                    unsigned layer) {
    std::vector<uint32_t> seen;
    for (const Cand& c : cands) seen.push_back(c.id);
    seen.push_back(base_id);
    std::sort(seen.begin(), seen.end());
    std::vector<Cand> out = cands;
    std::vector<uint32_t> list;
    for (const Cand& c : cands) {
        g.read(c.id, layer, list);
        for (uint32_t nb : list) {
            auto it = std::lower_bound(seen.begin(), seen.end(), nb);
            if (it != seen.end() && *it == nb) continue;
            seen.insert(it, nb);
            out.push_back(Cand{g.dist(base, nb), nb});
        }
    }
    std::sort(out.begin(), out.end(), CandLess());
    return out;
}

// select_neighbors (build.rs:153-196): simple, or the heuristic.
std::vector<uint32_t> select_neighbors(Graph& g, uint32_t base_id, const float* base, const std::vector<Cand>& cands,
                                       size_t m, unsigned layer) {
    std::vector<uint32_t> out;
    if (g.selection == 0) {
        for (size_t i = 0; i < cands.size() && i < m; ++i) out.push_back(cands[i].id);
        return out;
    }
    std::vector<Cand> extended;
    const std::vector<Cand>* pool = &cands;
    if (g.extend) {
        extended = extend_candidates(g, base_id, base, cands, layer);
        pool = &extended;
    }
    std::vector<Cand> selected, discarded;
    for (const Cand& c : *pool) {
        if (selected.size() >= m) break;
        const float* v = g.vec(c.id);
        bool diverse = true;
        for (const Cand& s : selected)
            if (!(metric_distance(g.metric, v, g.vec(s.id), g.dim) >= c.d)) {
                diverse = false;
                break;
            }
        if (diverse) selected.push_back(c);
        else if (g.keep) discarded.push_back(c);
    }
    const size_t room = m - selected.size();
    for (size_t i = 0; i < discarded.size() && i < room; ++i) selected.push_back(discarded[i]);
    for (const Cand& c : selected) out.push_back(c.id);
    return out;
}

// write_shrunk (build.rs:136-151); the caller holds the node's lock.
void write_shrunk(Graph& g, uint32_t node, const std::vector<uint32_t>& ids, unsigned layer) {
    const uint32_t cap = g.capacity(layer);
    if (ids.size() <= cap) {
        g.set(node, layer, ids);
        return;
    }
    const float* base = g.vec(node);
    std::vector<Cand> cands;
    for (uint32_t c : ids) cands.push_back(Cand{g.dist(base, c), c});
    std::sort(cands.begin(), cands.end(), CandLess());
    g.set(node, layer, select_neighbors(g, node, base, cands, cap, layer));
}

// install_own_neighbors (build.rs:100-117).
void install_own(Graph& g, uint32_t id, const std::vector<uint32_t>& selected, unsigned layer) {
    std::lock_guard<std::mutex> lock(g.locks[id]);
    std::vector<uint32_t> merged;
    g.read(id, layer, merged);
    if (merged.empty()) {
        g.set(id, layer, selected);
        return;
    }
    for (uint32_t nb : selected)
        if (std::find(merged.begin(), merged.end(), nb) == merged.end()) merged.push_back(nb);
    write_shrunk(g, id, merged, layer);
}

// connect (build.rs:121-132).
void connect(Graph& g, uint32_t node, uint32_t fresh, unsigned layer) {
    std::lock_guard<std::mutex> lock(g.locks[node]);
    std::vector<uint32_t> cur;
    g.read(node, layer, cur);
    if (std::find(cur.begin(), cur.end(), fresh) != cur.end() || g.try_push(node, layer, fresh)) return;
    cur.push_back(fresh);
    write_shrunk(g, node, cur, layer);
}

// link (build.rs:40-96).
void link(Graph& g, BuildScratch& sc, uint32_t id) {
    const unsigned level = g.levels[id];
    const float* q = g.vec(id);
    uint64_t entry = g.entry.load(std::memory_order_acquire);
    std::unique_lock<std::mutex> promotion;
    if (entry == kNoEntry || level > unsigned(entry >> 32)) {
        std::unique_lock<std::mutex> guard(g.promotion);
        entry = g.entry.load(std::memory_order_acquire);
        if (entry == kNoEntry) {
            g.entry.store((uint64_t(level) << 32) | id, std::memory_order_release);
            return;
        }
        if (level > unsigned(entry >> 32)) promotion = std::move(guard);
    }
    const uint32_t entry_id = uint32_t(entry);
    const unsigned top = unsigned(entry >> 32);
    Cand ep{g.dist(q, entry_id), entry_id};
    for (unsigned layer = top; layer > level; --layer) ep = build_greedy(g, sc, ep, layer, q);
    const size_t ef = std::max<size_t>(g.efc, g.m);
    std::vector<Cand> eps{ep};
    for (int layer = int(std::min(level, top)); layer >= 0; --layer) {
        std::vector<Cand> found = build_search_layer(g, sc, eps, ef, unsigned(layer), q, id);
        std::vector<uint32_t> selected = select_neighbors(g, id, q, found, g.m, unsigned(layer));
        install_own(g, id, selected, unsigned(layer));
        for (uint32_t nb : selected) connect(g, nb, id, unsigned(layer));
        if (!found.empty()) eps = std::move(found);
    }
    if (promotion.owns_lock()) g.entry.store((uint64_t(level) << 32) | id, std::memory_order_release);
}

// Format v1 writer (src/hnsw/io.rs:102-178), CRC-32 trailer.
std::vector<uint8_t> write_v1(Graph& g, const std::vector<uint8_t>& deleted) {
    std::vector<uint8_t> out;
    auto put = [&](const void* p, size_t k) {
        const uint8_t* b = static_cast<const uint8_t*>(p);
        out.insert(out.end(), b, b + k);
    };
    auto put32 = [&](uint32_t v) { put(&v, 4); };
    put("HNSWIDX\0", 8);
    put32(1);
    const uint8_t tags[4] = {uint8_t(g.metric), uint8_t(g.selection),
                             uint8_t(g.selection ? (uint8_t(g.extend) | (uint8_t(g.keep) << 1)) : 0), 0};
    put(tags, 4);
    put32(uint32_t(g.dim));
    put32(g.m);
    put32(g.m0);
    put32(g.efc);
    put(&g.ml, 8);
    put(&g.seed, 8);
    put32(g.n);
    const uint64_t e = g.entry.load();
    put32(e == kNoEntry ? 0xFFFFFFFFu : uint32_t(e));
    put(g.keys.data(), g.keys.size() * 8);
    put(g.levels.data(), g.levels.size());
    put(deleted.data(), deleted.size());
    put(g.vectors.data(), g.vectors.size() * 4);
    std::vector<uint32_t> list;
    for (uint32_t id = 0; id < g.n; ++id)
        for (unsigned layer = 0; layer <= g.levels[id]; ++layer) {
            g.read(id, layer, list);
            put32(uint32_t(list.size()));
            put(list.data(), list.size() * 4);
        }
    put32(crc32(out.data(), out.size()));
    return out;
}
}  // namespace

extern "C" {

// ---- kernels ----
float orc_dot(const float* a, const float* b, size_t n) { return k_dot(a, b, n); }
float orc_l2(const float* a, const float* b, size_t n) { return k_l2(a, b, n); }
float orc_dot_portable(const float* a, const float* b, size_t n) { return dot_avx2order_portable(a, b, n); }
float orc_l2_portable(const float* a, const float* b, size_t n) { return l2_avx2order_portable(a, b, n); }
float orc_dot_scalar(const float* a, const float* b, size_t n) { return dot_scalar(a, b, n); }
float orc_l2_scalar(const float* a, const float* b, size_t n) { return l2_scalar(a, b, n); }
float orc_distance(int metric, const float* a, const float* b, size_t n) { return metric_distance(metric, a, b, n); }
int64_t orc_i8_dot(const int8_t* a, const int8_t* b, size_t n) { return i8_dot(a, b, n); }
int64_t orc_i8_l2(const int8_t* a, const int8_t* b, size_t n) { return i8_l2(a, b, n); }
void orc_sq_encode(const float* x, const float* offset, float scale, size_t dim, int8_t* out) {
    sq_encode(x, offset, scale, dim, out);
}
float orc_sq_distance(int metric, float scale, const int8_t* a, const int8_t* b, size_t n) {
    return sq_distance(metric, scale, a, b, n);
}
int32_t orc_prepare_query(int metric, const float* q, size_t dim, float* out) {
    return prepare_query(metric, q, dim, out);
}
uint32_t orc_crc32(const uint8_t* p, size_t n) { return crc32(p, n); }
int orc_have_avx2() { return have_avx2() ? 1 : 0; }

// ---- generator ----
void orc_splitmix(uint64_t seed, uint64_t* out, size_t n) {
    SplitMix64 r{seed};
    for (size_t i = 0; i < n; ++i) out[i] = r.next();
}
// Dataset::gaussian (src/synthetic.rs:81-92): one stream, base then queries.
void orc_gaussian(size_t nb, size_t nq, size_t dim, uint64_t seed, float* base, float* queries) {
    SplitMix64 r{seed};
    for (size_t i = 0; i < nb * dim; ++i) base[i] = float(r.gaussian());
    for (size_t i = 0; i < nq * dim; ++i) queries[i] = float(r.gaussian());
}
// Dataset::clustered (src/synthetic.rs:102-124) with the spread as a parameter.
void orc_clustered(size_t nb, size_t nq, size_t dim, size_t clusters, double spread, uint64_t seed,
                   float* base, float* queries) {
    SplitMix64 r{seed};
    std::vector<double> centers(clusters * dim);
    for (auto& c : centers) c = r.gaussian();
    auto sample = [&](size_t count, float* out) {
        for (size_t p = 0; p < count; ++p) {
            size_t c = size_t(r.below(clusters));
            for (size_t j = 0; j < dim; ++j) out[p * dim + j] = float(centers[c * dim + j] + spread * r.gaussian());
        }
    };
    sample(nb, base);
    sample(nq, queries);
}


// ---- construction ----
// HnswIndex::insert_batch into an empty index (src/hnsw/mod.rs:318-349) of
// n rows with keys, then to_bytes. threads == 1 links the nodes in id order
// (the same graph as n calls of insert); threads != 1 links them
// concurrently (0: every core), whose graph depends on scheduling, as the
// reference's does (mod.rs:306-312). deleted_keys (count nd) are then
// removed (tombstoned). Returns the file size and writes it to *out
// (orc_free_bytes releases it), or 0 when a row fails validation.
size_t orc_build(size_t dim, int metric, uint32_t m, uint32_t m0, uint32_t efc, double ml, int selection,
                 int extend, int keep, uint64_t seed, const uint64_t* keys, const float* vectors, size_t n,
                 const uint64_t* deleted_keys, size_t nd, int threads, uint8_t** out) {
    *out = nullptr;
    Graph g;
    g.dim = dim;
    g.metric = metric;
    g.m = m;
    g.m0 = m0;
    g.efc = efc;
    g.ml = ml;
    g.selection = selection;
    g.extend = extend != 0;
    g.keep = keep != 0;
    g.seed = seed;
    g.n = uint32_t(n);
    g.vectors.resize(n * dim);
    for (size_t i = 0; i < n; ++i)  // prepare_batch (src/vector.rs:55-88)
        if (prepare_query(metric, vectors + i * dim, dim, g.vectors.data() + i * dim) != OK) return 0;
    g.keys.assign(keys, keys + n);
    g.levels.resize(n);
    g.up_off.resize(n);
    size_t up = 0;
    for (uint32_t id = 0; id < n; ++id) {
        g.levels[id] = sample_level(seed, id, ml);
        g.up_off[id] = up;
        up += size_t(g.levels[id]) * (m + 1);
    }
    g.l0 = std::vector<std::atomic<uint32_t>>(n * (m0 + 1));
    g.upper = std::vector<std::atomic<uint32_t>>(up);
    g.locks = std::vector<std::mutex>(n);
    if (threads == 1) {
        BuildScratch sc;
        for (uint32_t id = 0; id < n; ++id) link(g, sc, id);
    } else {
        BuildScratch first;
        if (n) link(g, first, 0);  // link_parallel: the first node alone sets the entry point
        const int nt = threads > 0 ? threads : int(std::max(1u, std::thread::hardware_concurrency()));
        std::atomic<uint32_t> next{1};
        std::vector<std::thread> pool;
        for (int t = 0; t < nt; ++t)
            pool.emplace_back([&] {
                BuildScratch sc;
                for (;;) {
                    const uint32_t id = next.fetch_add(1);
                    if (id >= n) break;
                    link(g, sc, id);
                }
            });
        for (auto& th : pool) th.join();
    }
    std::vector<uint8_t> deleted(n, 0);
    for (size_t j = 0; j < nd; ++j)
        for (uint32_t id = 0; id < n; ++id)
            if (g.keys[id] == deleted_keys[j] && !deleted[id]) {
                deleted[id] = 1;
                break;
            }
    std::vector<uint8_t> bytes = write_v1(g, deleted);
    *out = static_cast<uint8_t*>(std::malloc(bytes.size()));
    std::memcpy(*out, bytes.data(), bytes.size());
    return bytes.size();
}
void orc_free_bytes(uint8_t* p) { std::free(p); }

// Mixture with the base (and the centers) from base_seed and the queries
// from query_seed: the draw order of Dataset::clustered (src/synthetic.rs:
// 102-124: the centers, then per point next_below and dim Gaussians), with
// the spread as a parameter and the query points on their own stream.
void orc_mixture_split(size_t nb, size_t nq, size_t dim, size_t clusters, double spread, uint64_t base_seed,
                       uint64_t query_seed, float* base, float* queries) {
    SplitMix64 r{base_seed};
    std::vector<double> centers(clusters * dim);
    for (auto& c : centers) c = r.gaussian();
    auto sample = [&](SplitMix64& g, size_t count, float* out) {
        for (size_t p = 0; p < count; ++p) {
            const size_t c = size_t(g.below(clusters));
            for (size_t j = 0; j < dim; ++j) out[p * dim + j] = float(centers[c * dim + j] + spread * g.gaussian());
        }
    };
    sample(r, nb, base);
    SplitMix64 q{query_seed};
    sample(q, nq, queries);
}

// ---- index ----
void* orc_index_load(const uint8_t* p, size_t len) {
    if (len < 60 || std::memcmp(p, "HNSWIDX\0", 8) != 0) return nullptr;
    uint32_t stored;
    std::memcpy(&stored, p + len - 4, 4);
    if (crc32(p, len - 4) != stored) return nullptr;
    Rd r{p, len - 4, 8};
    auto* ix = new Index();
    if (r.get<uint32_t>() != 1) { delete ix; return nullptr; }
    ix->metric = r.get<uint8_t>();
    r.get<uint8_t>();
    r.get<uint8_t>();
    ix->quantized = r.get<uint8_t>() == 1;
    ix->dim = r.get<uint32_t>();
    ix->m = r.get<uint32_t>();
    ix->m0 = r.get<uint32_t>();
    r.get<uint32_t>();
    r.get<double>();
    r.get<uint64_t>();
    ix->n = r.get<uint32_t>();
    ix->entry = r.get<uint32_t>();
    size_t n = ix->n, dim = ix->dim;
    const uint8_t* kb = r.take(n * 8);
    const uint8_t* lb = r.take(n);
    const uint8_t* fb = r.take(n);
    const uint8_t* vb = r.take(n * dim * 4);
    if (!r.ok) { delete ix; return nullptr; }
    ix->keys.resize(n);
    std::memcpy(ix->keys.data(), kb, n * 8);
    ix->levels.assign(lb, lb + n);
    ix->deleted.assign(fb, fb + n);
    ix->vectors.resize(n * dim);
    std::memcpy(ix->vectors.data(), vb, n * dim * 4);
    ix->l0.assign(n * (ix->m0 + 1), 0);
    ix->upper.resize(n);
    for (size_t id = 0; id < n; ++id) {
        ix->top = std::max(ix->top, ix->levels[id]);
        ix->upper[id].assign(size_t(ix->levels[id]) * (ix->m + 1), 0);
        for (unsigned layer = 0; layer <= ix->levels[id]; ++layer) {
            uint32_t cnt = r.get<uint32_t>();
            uint32_t cap = layer == 0 ? ix->m0 : ix->m;
            if (!r.ok || cnt > cap) { delete ix; return nullptr; }
            uint32_t* blk = layer == 0 ? ix->l0.data() + id * (ix->m0 + 1)
                                       : ix->upper[id].data() + (layer - 1) * (ix->m + 1);
            blk[0] = cnt;
            for (uint32_t j = 0; j < cnt; ++j) blk[1 + j] = r.get<uint32_t>();
        }
    }
    if (ix->quantized) {
        ix->offset.resize(dim);
        for (size_t j = 0; j < dim; ++j) ix->offset[j] = r.get<float>();
        ix->scale = r.get<float>();
        ix->codes.resize(n * dim);
        // Codes are re-derived from offsets and scale (src/hnsw/mod.rs:769-775).
        for (size_t id = 0; id < n; ++id)
            sq_encode(ix->vec(uint32_t(id)), ix->offset.data(), ix->scale, dim, ix->codes.data() + id * dim);
    }
    if (!r.ok || r.pos != r.n) { delete ix; return nullptr; }
    for (size_t id = 0; id < n; ++id) ix->live += ix->deleted[id] ? 0 : 1;
    if (n == 0) ix->entry = 0xFFFFFFFFu;
    return ix;
}

void orc_index_free(void* ix) { delete static_cast<Index*>(ix); }
uint32_t orc_index_nodes(void* ix) { return static_cast<Index*>(ix)->n; }
uint32_t orc_index_dim(void* ix) { return static_cast<Index*>(ix)->dim; }
int orc_index_metric(void* ix) { return static_cast<Index*>(ix)->metric; }
const int8_t* orc_index_codes(void* ix) { return static_cast<Index*>(ix)->codes.data(); }

// HnswIndex::search_batch / search_with / search_filtered
// (src/hnsw/mod.rs:412-536). `filter_bits` (optional) is a key bitmap of
// `filter_nbits` bits, shared by all queries when filter_stride == 0, else
// query i uses filter_bits + i*filter_stride (in u64 words). Outputs are
// nq*k arrays; counts[i] results for query i. Per-query counters (optional):
// stats[4*i + {0,1,2,3}] = layer-0 distances, layer-0 expansions, upper-layer
// distances, upper-layer list reads.
void orc_search_batch(void* handle, const float* queries, size_t nq, size_t k, const size_t* ks,
                      size_t ef, const size_t* efs, int quantized, const uint64_t* filter_bits,
                      uint64_t filter_nbits, size_t filter_stride, const uint8_t* use_filter,
                      uint64_t* out_keys, float* out_dist, uint32_t* counts, int32_t* status,
                      uint64_t* stats, int threads, size_t out_stride, int filter_by_node) {
    const Index& ix = *static_cast<Index*>(handle);
    int nt = threads <= 0 ? int(std::max(1u, std::thread::hardware_concurrency())) : threads;
    std::vector<Scratch> scratch(static_cast<size_t>(nt));
    if (out_stride == 0) out_stride = k;
    parallel_for(nq, nt, [&](int t, size_t i) {
        Filter f;
        if (filter_bits && (!use_filter || use_filter[i])) {
            f.bits = filter_bits + (filter_stride ? i * filter_stride : 0);
            f.nbits = filter_nbits;
            f.by_node = filter_by_node != 0;
        }
        std::vector<Hit> hits;
        Stats st;
        size_t ki = ks ? ks[i] : k, efi = efs ? efs[i] : ef;
        status[i] = search_one(ix, scratch[size_t(t)], queries + i * ix.dim, ki, efi, quantized != 0, f, hits, st);
        counts[i] = uint32_t(hits.size());
        for (size_t j = 0; j < hits.size(); ++j) {
            out_keys[i * out_stride + j] = hits[j].key;
            out_dist[i * out_stride + j] = hits[j].d;
        }
        if (stats) {
            stats[4 * i + 0] = st.dist0;
            stats[4 * i + 1] = st.exp0;
            stats[4 * i + 2] = st.dist_up;
            stats[4 * i + 3] = st.exp_up;
        }
    });
}

// BruteForceIndex::search_filtered / search_batch (src/brute.rs:122-180) over
// rows already prepared (unit length for cosine, src/vector.rs:50-66): a
// bounded max-heap of (total_cmp distance, key), into_sorted_vec ascending.
// With `filter_bits`, a row is scored only when its bit is set (bit = key, or
// row index with by_row): query i uses filter_bits + i * filter_stride words
// (stride 0: one shared bitmap), as search_filtered's closure does.
void orc_brute_filtered(int metric, const float* base, const uint64_t* keys, size_t nb, size_t dim,
                        const float* queries, size_t nq, size_t k, const uint64_t* filter_bits, uint64_t filter_nbits,
                        size_t filter_stride, int by_row, uint64_t* out_keys, float* out_dist, uint32_t* counts,
                        int32_t* status, int threads) {
    parallel_for(nq, threads, [&](int, size_t i) {
        std::vector<float> q(dim);
        status[i] = prepare_query(metric, queries + i * dim, dim, q.data());
        counts[i] = 0;
        if (status[i] != OK || k == 0) return;
        // At most `len` results, whatever k asks for (src/brute.rs:141-142).
        size_t kk = std::min(k, nb);
        auto less = [](const Hit& a, const Hit& b) { return hit_less(a, b); };
        std::priority_queue<Hit, std::vector<Hit>, decltype(less)> heap(less);
        const uint64_t* fb = filter_bits ? filter_bits + i * filter_stride : nullptr;
        for (size_t r = 0; r < nb; ++r) {
            const uint64_t key = keys ? keys[r] : uint64_t(r);
            if (fb) {
                const uint64_t bit = by_row ? uint64_t(r) : key;
                if (bit >= filter_nbits || !((fb[bit >> 6] >> (bit & 63)) & 1)) continue;
            }
            Hit h{key, metric_distance(metric, q.data(), base + r * dim, dim)};
            if (heap.size() < kk) heap.push(h);
            else if (hit_less(h, heap.top())) {
                heap.pop();
                heap.push(h);
            }
        }
        size_t c = heap.size();
        counts[i] = uint32_t(c);
        for (size_t j = c; j-- > 0;) {
            out_keys[i * k + j] = heap.top().key;
            out_dist[i * k + j] = heap.top().d;
            heap.pop();
        }
    });
}

void orc_brute_batch(int metric, const float* base, const uint64_t* keys, size_t nb, size_t dim,
                     const float* queries, size_t nq, size_t k, uint64_t* out_keys, float* out_dist,
                     uint32_t* counts, int32_t* status, int threads) {
    orc_brute_filtered(metric, base, keys, nb, dim, queries, nq, k, nullptr, 0, 0, 0, out_keys, out_dist, counts,
                       status, threads);
}

// Double-precision scoring for the precision study of brute force: exact
// top-k by (f64 distance, key). Used as the FP64 oracle.
void orc_brute_f64(int metric, const float* base, size_t nb, size_t dim, const float* queries, size_t nq,
                   size_t k, uint64_t* out_keys, double* out_dist, int threads) {
    parallel_for(nq, threads, [&](int, size_t i) {
        const float* q = queries + i * dim;
        std::vector<std::pair<double, uint64_t>> best;
        best.reserve(k + 1);
        auto cmp = [](const std::pair<double, uint64_t>& a, const std::pair<double, uint64_t>& b) {
            return a.first != b.first ? a.first < b.first : a.second < b.second;
        };
        std::priority_queue<std::pair<double, uint64_t>, std::vector<std::pair<double, uint64_t>>, decltype(cmp)> heap(cmp);
        for (size_t r = 0; r < nb; ++r) {
            const float* x = base + r * dim;
            double s = 0.0;
            if (metric == L2) {
                for (size_t j = 0; j < dim; ++j) {
                    double d = double(q[j]) - double(x[j]);
                    s += d * d;
                }
            } else {
                for (size_t j = 0; j < dim; ++j) s += double(q[j]) * double(x[j]);
                s = metric == IP ? -s : 1.0 - s;
            }
            std::pair<double, uint64_t> h{s, uint64_t(r)};
            if (heap.size() < k) heap.push(h);
            else if (cmp(h, heap.top())) {
                heap.pop();
                heap.push(h);
            }
        }
        size_t c = heap.size();
        for (size_t j = c; j-- > 0;) {
            out_keys[i * k + j] = heap.top().second;
            out_dist[i * k + j] = heap.top().first;
            heap.pop();
        }
    });
}

// eval::recall_at_k (src/eval.rs:25-47) over fixed-stride key arrays.
double orc_recall_at_k(const uint64_t* truth, const uint32_t* truth_counts, size_t truth_stride,
                       const uint64_t* found, const uint32_t* found_counts, size_t found_stride, size_t nq,
                       size_t k) {
    size_t hits = 0, expected = 0;
    for (size_t i = 0; i < nq; ++i) {
        size_t tn = std::min<size_t>(k, truth_counts[i]), fn = std::min<size_t>(k, found_counts[i]);
        expected += tn;
        for (size_t a = 0; a < fn; ++a)
            for (size_t b = 0; b < tn; ++b)
                if (found[i * found_stride + a] == truth[i * truth_stride + b]) {
                    ++hits;
                    break;
                }
    }
    return expected == 0 ? 1.0 : double(hits) / double(expected);
}

}  // extern "C"
