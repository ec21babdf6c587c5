// Host-side index: validating loader, writer, construction, generators.
// Compiled with -ffp-contract=off so that every rounding matches the
// reference (Rust never contracts a*b+c; FMAs below are explicit).
#include "host_index.hpp"

#include <immintrin.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <queue>
#include <thread>
#include <unordered_set>

#include "hnsw_gpu.h"

namespace hnswgpu {

// ---------------------------------------------------------------------------
// Parameters
// ---------------------------------------------------------------------------
Params default_params(uint32_t m) {
    Params p;
    p.m = m;
    p.m0 = m > 0x7FFFFFFFu ? 0xFFFFFFFFu : 2 * m;  // saturating_mul(2)
    p.ef_construction = 200;
    p.level_multiplier = 1.0 / std::log(double(m));
    p.selection = 1;
    p.extend_candidates = p.keep_pruned = false;
    p.seed = 0;
    return p;
}

const char* validate_params(const Params& p) {
    if (p.m < 2 || p.m > 512) return "m";
    if (p.m0 < p.m || p.m0 > 2048) return "m0";
    if (p.ef_construction < 1 || p.ef_construction > 65536) return "ef_construction";
    if (!(std::isfinite(p.level_multiplier) && p.level_multiplier > 0.0 && p.level_multiplier <= 10.0))
        return "level_multiplier";
    return "";
}

// ---------------------------------------------------------------------------
// CRC-32, slicing-by-8 (Kounavis & Berry), reflected polynomial 0xEDB88320.
// ---------------------------------------------------------------------------
namespace {
struct CrcTables {
    uint32_t t[8][256];
    CrcTables() {
        for (uint32_t i = 0; i < 256; ++i) {
            uint32_t c = i;
            for (int k = 0; k < 8; ++k) c = (c & 1) ? (c >> 1) ^ 0xEDB88320u : c >> 1;
            t[0][i] = c;
        }
        for (int s = 1; s < 8; ++s)
            for (int i = 0; i < 256; ++i) t[s][i] = (t[s - 1][i] >> 8) ^ t[0][t[s - 1][i] & 0xFF];
    }
};
const CrcTables& crc_tables() {
    static CrcTables tables;
    return tables;
}
}  // namespace

uint32_t crc32(const uint8_t* p, size_t n) {
    const auto& T = crc_tables().t;
    uint32_t c = 0xFFFFFFFFu;
    size_t i = 0;
    for (; i + 8 <= n; i += 8) {
        uint32_t lo;
        std::memcpy(&lo, p + i, 4);
        lo ^= c;
        c = T[7][lo & 0xFF] ^ T[6][(lo >> 8) & 0xFF] ^ T[5][(lo >> 16) & 0xFF] ^ T[4][lo >> 24] ^
            T[3][p[i + 4]] ^ T[2][p[i + 5]] ^ T[1][p[i + 6]] ^ T[0][p[i + 7]];
    }
    for (; i < n; ++i) c = (c >> 8) ^ T[0][(c ^ p[i]) & 0xFF];
    return ~c;
}

// ---------------------------------------------------------------------------
// f32 kernels (AVX2 backend order, src/kernels/x86.rs:19-131).
// ---------------------------------------------------------------------------
namespace {
inline float hsum8(const float* v) { return ((v[0] + v[4]) + (v[1] + v[5])) + ((v[2] + v[6]) + (v[3] + v[7])); }

__attribute__((target("avx2,fma"))) float dot_avx2(const float* a, const float* b, size_t len) {
    __m256 c0 = _mm256_setzero_ps(), c1 = _mm256_setzero_ps(), c2 = _mm256_setzero_ps(), c3 = _mm256_setzero_ps();
    size_t i = 0;
    for (; i + 32 <= len; i += 32) {
        c0 = _mm256_fmadd_ps(_mm256_loadu_ps(a + i), _mm256_loadu_ps(b + i), c0);
        c1 = _mm256_fmadd_ps(_mm256_loadu_ps(a + i + 8), _mm256_loadu_ps(b + i + 8), c1);
        c2 = _mm256_fmadd_ps(_mm256_loadu_ps(a + i + 16), _mm256_loadu_ps(b + i + 16), c2);
        c3 = _mm256_fmadd_ps(_mm256_loadu_ps(a + i + 24), _mm256_loadu_ps(b + i + 24), c3);
    }
    for (; i + 8 <= len; i += 8) c0 = _mm256_fmadd_ps(_mm256_loadu_ps(a + i), _mm256_loadu_ps(b + i), c0);
    float v[8];
    _mm256_storeu_ps(v, _mm256_add_ps(_mm256_add_ps(c0, c1), _mm256_add_ps(c2, c3)));
    float s = hsum8(v);
    for (; i < len; ++i) s += a[i] * b[i];
    return s;
}
__attribute__((target("avx2,fma"))) float l2_avx2(const float* a, const float* b, size_t len) {
    __m256 c0 = _mm256_setzero_ps(), c1 = _mm256_setzero_ps(), c2 = _mm256_setzero_ps(), c3 = _mm256_setzero_ps();
    size_t i = 0;
    for (; i + 32 <= len; i += 32) {
        __m256 d0 = _mm256_sub_ps(_mm256_loadu_ps(a + i), _mm256_loadu_ps(b + i));
        __m256 d1 = _mm256_sub_ps(_mm256_loadu_ps(a + i + 8), _mm256_loadu_ps(b + i + 8));
        __m256 d2 = _mm256_sub_ps(_mm256_loadu_ps(a + i + 16), _mm256_loadu_ps(b + i + 16));
        __m256 d3 = _mm256_sub_ps(_mm256_loadu_ps(a + i + 24), _mm256_loadu_ps(b + i + 24));
        c0 = _mm256_fmadd_ps(d0, d0, c0);
        c1 = _mm256_fmadd_ps(d1, d1, c1);
        c2 = _mm256_fmadd_ps(d2, d2, c2);
        c3 = _mm256_fmadd_ps(d3, d3, c3);
    }
    for (; i + 8 <= len; i += 8) {
        __m256 d = _mm256_sub_ps(_mm256_loadu_ps(a + i), _mm256_loadu_ps(b + i));
        c0 = _mm256_fmadd_ps(d, d, c0);
    }
    float v[8];
    _mm256_storeu_ps(v, _mm256_add_ps(_mm256_add_ps(c0, c1), _mm256_add_ps(c2, c3)));
    float s = hsum8(v);
    for (; i < len; ++i) {
        float d = a[i] - b[i];
        s += d * d;
    }
    return s;
}
float dot_generic(const float* a, const float* b, size_t len) {
    float acc[4][8] = {};
    size_t i = 0;
    for (; i + 32 <= len; i += 32)
        for (int c = 0; c < 4; ++c)
            for (int l = 0; l < 8; ++l) acc[c][l] = std::fmaf(a[i + 8 * c + l], b[i + 8 * c + l], acc[c][l]);
    for (; i + 8 <= len; i += 8)
        for (int l = 0; l < 8; ++l) acc[0][l] = std::fmaf(a[i + l], b[i + l], acc[0][l]);
    float v[8];
    for (int l = 0; l < 8; ++l) v[l] = (acc[0][l] + acc[1][l]) + (acc[2][l] + acc[3][l]);
    float s = hsum8(v);
    for (; i < len; ++i) s += a[i] * b[i];
    return s;
}
float l2_generic(const float* a, const float* b, size_t len) {
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
    float s = hsum8(v);
    for (; i < len; ++i) {
        float d = a[i] - b[i];
        s += d * d;
    }
    return s;
}
bool cpu_avx2() {
    static const bool ok = __builtin_cpu_supports("avx2") && __builtin_cpu_supports("fma");
    return ok;
}
}  // namespace

float dot_ref(const float* a, const float* b, size_t n) { return cpu_avx2() ? dot_avx2(a, b, n) : dot_generic(a, b, n); }
float l2_ref(const float* a, const float* b, size_t n) { return cpu_avx2() ? l2_avx2(a, b, n) : l2_generic(a, b, n); }
float metric_distance(int metric, const float* a, const float* b, size_t n) {
    switch (metric) {
        case HNSW_METRIC_L2: return l2_ref(a, b, n);
        case HNSW_METRIC_INNER_PRODUCT: return -dot_ref(a, b, n);
        default: return 1.0f - dot_ref(a, b, n);
    }
}

int check_vector(const float* v, size_t dim, double* norm_sq) {
    double s = 0.0;
    for (size_t i = 0; i < dim; ++i) {
        if (!std::isfinite(v[i])) return HNSW_ERR_NON_FINITE_VECTOR;
        s += double(v[i]) * double(v[i]);
    }
    if (s > double(3.40282346638528859812e+38F) / 8.0) return HNSW_ERR_NON_FINITE_VECTOR;
    *norm_sq = s;
    return HNSW_OK;
}

// ---------------------------------------------------------------------------
// Loader (src/hnsw/io.rs:236-540)
// ---------------------------------------------------------------------------
namespace {

constexpr uint8_t kMagic[8] = {'H', 'N', 'S', 'W', 'I', 'D', 'X', 0};
constexpr size_t kHeaderLen = 56, kTrailerLen = 4;

Err fail(int status, const char* what = "") {
    Err e;
    e.status = status;
    e.what = what;
    return e;
}
Err invalid(const char* what) { return fail(HNSW_ERR_FORMAT_INVALID, what); }

struct Reader {
    const uint8_t* buf;
    size_t len, pos;
    bool take(size_t n, const uint8_t** out) {
        if (n > len - pos) return false;
        *out = buf + pos;
        pos += n;
        return true;
    }
    template <class T>
    bool get(T* v) {
        const uint8_t* p;
        if (!take(sizeof(T), &p)) return false;
        std::memcpy(v, p, sizeof(T));
        return true;
    }
};

// key_map_heap_bytes (src/hnsw/mod.rs:781-786): hashbrown buckets of (u64, u32) + 1 control byte.
uint64_t key_map_heap_bytes(uint64_t capacity) {
    unsigned __int128 want = (unsigned __int128)capacity * 8 / 7;
    uint64_t buckets;
    if (want > (uint64_t(1) << 63)) buckets = ~0ull;
    else {
        buckets = 1;
        while (buckets < uint64_t(want)) buckets <<= 1;
    }
    unsigned __int128 r = (unsigned __int128)buckets * 17;
    return r > ~0ull ? ~0ull : uint64_t(r);
}

uint64_t sat_add(uint64_t a, uint64_t b) { return a > ~0ull - b ? ~0ull : a + b; }
uint64_t sat_mul(uint64_t a, uint64_t b) {
    unsigned __int128 r = (unsigned __int128)a * b;
    return r > ~0ull ? ~0ull : uint64_t(r);
}

}  // namespace

// verify_envelope without the checksum (io.rs:278-305): magic, version,
// minimum length. *body_len is the length the CRC covers, *stored the CRC.
Err check_envelope(const uint8_t* bytes, size_t len, size_t* body_len, uint32_t* stored) {
    if (len < 12) {
        size_t pl = std::min<size_t>(len, 8);
        return fail(std::memcmp(bytes, kMagic, pl) == 0 ? HNSW_ERR_FORMAT_TRUNCATED : HNSW_ERR_FORMAT_BAD_MAGIC);
    }
    if (std::memcmp(bytes, kMagic, 8) != 0) return fail(HNSW_ERR_FORMAT_BAD_MAGIC);
    uint32_t version;
    std::memcpy(&version, bytes + 8, 4);
    if (version != 1) {
        Err e = fail(HNSW_ERR_FORMAT_UNSUPPORTED_VERSION);
        e.a = version;
        return e;
    }
    if (len < kHeaderLen + kTrailerLen) return fail(HNSW_ERR_FORMAT_TRUNCATED);
    *body_len = len - kTrailerLen;
    std::memcpy(stored, bytes + *body_len, 4);
    return Err();
}

Err invalid_field(const char* what) { return invalid(what); }

Err checksum_error(uint32_t stored, uint32_t computed) {
    Err e = fail(HNSW_ERR_FORMAT_CHECKSUM);
    e.a = stored;
    e.b = computed;
    return e;
}

// read_header, read_columns, scan_links and required_memory (io.rs:317-445)
// on a body whose checksum is verified: every check that needs no vector or
// list contents, in the reference's order, recording where each part lies.
Err scan_layout(const uint8_t* bytes, size_t body_len, uint64_t max_memory, FileLayout* out) {
    if (max_memory == 0) max_memory = std::max<uint64_t>(sat_mul(body_len + kTrailerLen, 64), uint64_t(64) << 20);
    Reader r{bytes, body_len, 12};
    const Err truncated = fail(HNSW_ERR_FORMAT_TRUNCATED);
    FileLayout& L = *out;
    L = FileLayout();
    L.body_len = body_len;

    // read_header (io.rs:317-361)
    uint8_t metric, sel, flags, qflag;
    if (!r.get(&metric)) return truncated;
    if (metric > 2) return invalid("metric");
    if (!r.get(&sel) || !r.get(&flags)) return truncated;
    Params p;
    if (sel == 0 && flags == 0) p.selection = 0;
    else if (sel == 1 && flags <= 3) {
        p.selection = 1;
        p.extend_candidates = (flags & 1) != 0;
        p.keep_pruned = (flags & 2) != 0;
    } else return invalid("neighbor selection");
    if (!r.get(&qflag)) return truncated;
    if (qflag > 1) return invalid("quantized flag");
    uint32_t dim, m, m0, efc, n, entry_id;
    double ml;
    uint64_t seed;
    if (!r.get(&dim)) return truncated;
    if (dim == 0 || dim > kMaxDim) return invalid("dimension");
    if (!r.get(&m) || !r.get(&m0) || !r.get(&efc) || !r.get(&ml) || !r.get(&seed)) return truncated;
    p.m = m;
    p.m0 = m0;
    p.ef_construction = efc;
    p.level_multiplier = ml;
    p.seed = seed;
    if (*validate_params(p)) return invalid("parameters");
    if (!r.get(&n)) return truncated;
    if (uint64_t(n) > kMaxNodes) return invalid("node count");
    if (!r.get(&entry_id)) return truncated;
    L.metric = metric;
    L.quantized = qflag != 0;
    L.params = p;
    L.dim = dim;
    L.n = n;
    L.entry_id = entry_id;

    // read_columns (io.rs:375-402)
    const uint8_t *kcol, *lcol, *fcol, *vcol;
    if (!r.take(size_t(n) * 8, &kcol) || !r.take(n, &lcol) || !r.take(n, &fcol)) return truncated;
    if (uint64_t(n) * 4 * dim > uint64_t(SIZE_MAX)) return truncated;
    if (!r.take(size_t(n) * 4 * dim, &vcol)) return truncated;
    for (uint32_t i = 0; i < n; ++i)
        if (lcol[i] > kMaxLevel) return invalid("node level");
    for (uint32_t i = 0; i < n; ++i)
        if (fcol[i] > 1) return invalid("tombstone flag");
    uint64_t level_sum = 0;
    for (uint32_t i = 0; i < n; ++i) level_sum += lcol[i];
    double expected = double(n) / std::expm1(1.0 / ml);
    if (double(level_sum) > 2.0 * expected + 1024.0) return invalid("implausible level distribution");
    L.keys = kcol;
    L.levels = lcol;
    L.dead = fcol;
    L.vectors = vcol;
    L.level_sum = level_sum;
    L.links_begin = r.pos;

    // scan_links (io.rs:407-419): walk without allocating (beyond one offset
    // per node, where the node's first list starts).
    {
        Reader s = r;
        L.node_off.resize(n);
        for (uint32_t i = 0; i < n; ++i) {
            L.node_off[i] = s.pos;
            for (unsigned layer = 0; layer <= lcol[i]; ++layer) {
                uint32_t count;
                if (!s.get(&count)) return truncated;
                uint32_t cap = layer == 0 ? m0 : m;
                if (count > cap) return invalid("neighbor count exceeds capacity");
                const uint8_t* skip;
                if (!s.take(size_t(count) * 4, &skip)) return truncated;
            }
        }
        L.links_end = s.pos;
    }
    // required_memory (io.rs:424-445); Mutex<()> is 1 byte, Box<[AtomicU32]> 16.
    uint64_t code = qflag ? dim : 0;
    uint64_t per_node = 4ull * dim + 8 + 1 + 1 + 1 + 16 + (uint64_t(m0) + 1) * 4 + code;
    uint64_t quantizer = qflag ? 4ull * dim : 0;
    uint64_t required = sat_add(sat_add(sat_add(sat_mul(n, per_node), sat_mul(level_sum, (uint64_t(m) + 1) * 4)),
                                        key_map_heap_bytes(n)),
                                quantizer);
    L.required = required;
    if (required > max_memory) {
        Err e = fail(HNSW_ERR_MEMORY_LIMIT_EXCEEDED);
        e.a = required;
        e.b = max_memory;
        return e;
    }
    return Err();
}

// The quantizer section and the trailing-bytes check (io.rs:487-515, after
// the lists), then the entry point (io.rs:517-540).
Err scan_tail(const uint8_t* bytes, const FileLayout& L, std::vector<float>* q_offset, float* q_scale) {
    Reader r{bytes, L.body_len, L.links_end};
    const Err truncated = fail(HNSW_ERR_FORMAT_TRUNCATED);
    if (L.quantized) {
        q_offset->resize(L.dim);
        const uint8_t* ob;
        if (!r.take(size_t(L.dim) * 4, &ob)) return truncated;
        std::memcpy(q_offset->data(), ob, size_t(L.dim) * 4);
        for (float o : *q_offset)
            if (!std::isfinite(o)) return invalid("quantizer offset");
        float scale;
        if (!r.get(&scale)) return truncated;
        if (!(std::isfinite(scale) && scale > 0.0f)) return invalid("quantizer");
        *q_scale = scale;
    }
    if (r.pos != r.len) return fail(HNSW_ERR_FORMAT_TRAILING_BYTES);
    return Err();
}

// The entry point check of finish (io.rs:517-540), after the key checks.
Err check_entry(const FileLayout& L, uint64_t* entry_word) {
    if (L.n == 0) {
        if (L.entry_id != kNoEntry) return invalid("entry point of an empty index");
        *entry_word = ~0ull;
        return Err();
    }
    const uint8_t top = *std::max_element(L.levels, L.levels + L.n);
    if (L.entry_id >= L.n || L.levels[L.entry_id] != top) return invalid("entry point");
    *entry_word = (uint64_t(top) << 32) | L.entry_id;
    return Err();
}

Err load_index(const uint8_t* bytes, size_t len, uint64_t max_memory, HostIndex* out, uint64_t* required_out) {
    size_t body_len = 0;
    uint32_t stored = 0;
    Err e = check_envelope(bytes, len, &body_len, &stored);
    if (e) return e;
    const uint32_t computed = crc32(bytes, body_len);
    if (stored != computed) return checksum_error(stored, computed);
    FileLayout L;
    e = scan_layout(bytes, body_len, max_memory, &L);
    if (required_out) *required_out = L.required;
    if (e) return e;
    Reader r{bytes, body_len, L.links_begin};
    const Err truncated = fail(HNSW_ERR_FORMAT_TRUNCATED);
    const uint32_t n = L.n, dim = L.dim, m0 = L.params.m0, m = L.params.m;
    const uint8_t *kcol = L.keys, *lcol = L.levels, *fcol = L.dead, *vcol = L.vectors;
    const uint8_t metric = L.metric;
    const Params p = L.params;

    // read_nodes (io.rs:448-485)
    HostIndex& ix = *out;
    ix = HostIndex();
    ix.dim = dim;
    ix.metric = metric;
    ix.params = p;
    ix.keys.resize(n);
    std::memcpy(ix.keys.data(), kcol, size_t(n) * 8);
    ix.vectors.resize(size_t(n) * dim);
    std::memcpy(ix.vectors.data(), vcol, size_t(n) * dim * 4);
    for (uint32_t i = 0; i < n; ++i) {
        double norm;
        if (check_vector(ix.vector(i), dim, &norm) != HNSW_OK) return invalid("vector out of range");
        if (metric == HNSW_METRIC_COSINE && std::fabs(norm - 1.0) > 1e-3)
            return invalid("cosine vector is not unit length");
    }
    ix.levels.assign(lcol, lcol + n);
    ix.deleted.assign(fcol, fcol + n);
    ix.l0.assign(size_t(n) * (m0 + 1), 0);
    ix.upper.resize(n);
    for (uint32_t i = 0; i < n; ++i) ix.upper[i].assign(size_t(lcol[i]) * (m + 1), 0);

    // read_links (io.rs:487-514)
    std::vector<uint32_t> nbrs, sorted;
    for (uint32_t id = 0; id < n; ++id)
        for (unsigned layer = 0; layer <= ix.levels[id]; ++layer) {
            uint32_t count;
            if (!r.get(&count)) return truncated;
            if (count > ix.capacity(layer)) return invalid("neighbor count exceeds capacity");
            nbrs.clear();
            for (uint32_t j = 0; j < count; ++j) {
                uint32_t nb;
                if (!r.get(&nb)) return truncated;
                bool valid = nb < n && nb != id && ix.levels[nb] >= layer;
                if (!valid) return invalid("neighbor id");
                nbrs.push_back(nb);
            }
            sorted = nbrs;
            std::sort(sorted.begin(), sorted.end());
            if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end())
                return invalid("duplicate neighbor id");
            uint32_t* blk = ix.block(id, layer);
            blk[0] = count;
            std::copy(nbrs.begin(), nbrs.end(), blk + 1);
        }
    e = scan_tail(bytes, L, &ix.q_offset, &ix.q_scale);
    if (e) return e;
    ix.quantized = L.quantized;

    // finish (io.rs:517-540)
    ix.key_to_id.reserve(n);
    for (uint32_t id = 0; id < n; ++id)
        if (!ix.deleted[id] && !ix.key_to_id.emplace(ix.keys[id], id).second) return invalid("duplicate live key");
    return check_entry(L, &ix.entry_word);
}

// ---------------------------------------------------------------------------
// Writer (src/hnsw/io.rs:103-169)
// ---------------------------------------------------------------------------
std::vector<uint8_t> write_index(const HostIndex& ix) {
    std::vector<uint8_t> out;
    size_t n = ix.node_count();
    out.reserve(64 + n * (8 + 2 + 4 * ix.dim + 4 * (ix.params.m0 + 1)));
    auto put = [&](const void* p, size_t k) {
        const uint8_t* b = static_cast<const uint8_t*>(p);
        out.insert(out.end(), b, b + k);
    };
    auto put32 = [&](uint32_t v) { put(&v, 4); };
    put(kMagic, 8);
    put32(1);
    uint8_t sel = ix.params.selection == 0 ? 0 : 1;
    uint8_t flags = sel ? uint8_t((ix.params.extend_candidates ? 1 : 0) | (ix.params.keep_pruned ? 2 : 0)) : 0;
    uint8_t hdr[4] = {uint8_t(ix.metric), sel, flags, uint8_t(ix.quantized ? 1 : 0)};
    put(hdr, 4);
    put32(ix.dim);
    put32(ix.params.m);
    put32(ix.params.m0);
    put32(ix.params.ef_construction);
    put(&ix.params.level_multiplier, 8);
    put(&ix.params.seed, 8);
    put32(uint32_t(n));
    put32(ix.has_entry() ? ix.entry_id() : kNoEntry);
    put(ix.keys.data(), n * 8);
    put(ix.levels.data(), n);
    put(ix.deleted.data(), n);
    put(ix.vectors.data(), n * ix.dim * 4);
    for (size_t id = 0; id < n; ++id)
        for (unsigned layer = 0; layer <= ix.levels[id]; ++layer) {
            const uint32_t* blk = ix.block(uint32_t(id), layer);
            uint32_t cnt = std::min(__atomic_load_n(blk, __ATOMIC_ACQUIRE), ix.capacity(layer));
            put32(cnt);
            put(blk + 1, size_t(cnt) * 4);
        }
    if (ix.quantized) {
        put(ix.q_offset.data(), ix.dim * 4);
        put(&ix.q_scale, 4);
    }
    uint32_t crc = crc32(out.data(), out.size());
    put32(crc);
    return out;
}

// ---------------------------------------------------------------------------
// Synthetic data (src/synthetic.rs:23-124)
// ---------------------------------------------------------------------------
namespace {
inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
struct SplitMix64 {
    uint64_t s;
    uint64_t next() { return mix64(s += 0x9E3779B97F4A7C15ULL); }
    double unit() { return double(next() >> 11) * (1.0 / double(1ULL << 53)); }
    uint64_t below(uint64_t n) { return uint64_t((unsigned __int128)next() * n >> 64); }
    double gaussian() {
        double u1 = 1.0 - unit();
        double u2 = unit();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};
}  // namespace

namespace {
constexpr uint64_t kGamma = 0x9E3779B97F4A7C15ULL;
// Runs f(begin, end) over [0, n) on all cores (for independent chunks).
template <class F>
void parallel_chunks(size_t n, F&& f) {
    const size_t threads = std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), n / 4096 + 1));
    if (threads == 1) {
        f(size_t(0), n);
        return;
    }
    std::vector<std::thread> pool;
    for (size_t t = 0; t < threads; ++t)
        pool.emplace_back([&, t] { f(n * t / threads, n * (t + 1) / threads); });
    for (auto& th : pool) th.join();
}
}  // namespace

// SplitMix64 is counter based: output i of the stream seeded with s is
// mix64(s + (i + 1) * gamma). Each chunk starts its own generator at its
// offset, so the parallel fill is bit-identical to one sequential stream.
void synthetic_gaussian(size_t nb, size_t nq, size_t dim, uint64_t seed, float* base, float* queries) {
    const size_t total = (nb + nq) * dim;
    parallel_chunks(total, [&](size_t b, size_t e) {
        SplitMix64 r{seed + uint64_t(2 * b) * kGamma};
        for (size_t i = b; i < e; ++i) {
            const float v = float(r.gaussian());
            if (i < nb * dim) base[i] = v;
            else queries[i - nb * dim] = v;
        }
    });
}

void synthetic_mixture(size_t nb, size_t nq, size_t dim, size_t clusters, double sigma, uint64_t seed, float* base,
                       float* queries) {
    SplitMix64 r{seed};
    std::vector<double> centers(clusters * dim);
    for (auto& c : centers) c = r.gaussian();
    auto sample = [&](size_t count, float* out) {
        for (size_t p = 0; p < count; ++p) {
            size_t c = size_t(r.below(clusters));
            for (size_t j = 0; j < dim; ++j) out[p * dim + j] = float(centers[c * dim + j] + sigma * r.gaussian());
        }
    };
    sample(nb, base);
    sample(nq, queries);
}

void synthetic_mixture_split(size_t nb, size_t nq, size_t dim, size_t clusters, double sigma, uint64_t base_seed,
                             uint64_t query_seed, float* base, float* queries) {
    SplitMix64 r{base_seed};
    std::vector<double> centers(clusters * dim);
    for (auto& c : centers) c = r.gaussian();
    // Each point consumes 1 + 2 * dim outputs (next_below, then dim Gaussians).
    const uint64_t per_point = 1 + 2 * uint64_t(dim);
    auto sample = [&](uint64_t stream_start, size_t count, float* out) {
        parallel_chunks(count, [&](size_t b, size_t e) {
            SplitMix64 g{stream_start + uint64_t(b) * per_point * kGamma};
            for (size_t p = b; p < e; ++p) {
                size_t c = size_t(g.below(clusters));
                for (size_t j = 0; j < dim; ++j) out[p * dim + j] = float(centers[c * dim + j] + sigma * g.gaussian());
            }
        });
    };
    sample(r.s, nb, base);
    sample(query_seed, nq, queries);
}

// ---------------------------------------------------------------------------
// Construction (src/hnsw/mod.rs:290-400, src/hnsw/build.rs:19-222)
// ---------------------------------------------------------------------------
namespace {


inline int32_t total_key(float f) {
    int32_t b;
    std::memcpy(&b, &f, 4);
    return b ^ int32_t(uint32_t(b >> 31) >> 1);
}
struct Cand {
    float d;
    uint32_t id;
};
inline bool cand_less(const Cand& a, const Cand& b) {
    int32_t ka = total_key(a.d), kb = total_key(b.d);
    return ka != kb ? ka < kb : a.id < b.id;
}
struct Less {
    bool operator()(const Cand& a, const Cand& b) const { return cand_less(a, b); }
};
struct Greater {
    bool operator()(const Cand& a, const Cand& b) const { return cand_less(b, a); }
};

struct SpinLock {
    std::atomic<uint8_t> f{0};
    void lock() {
        while (f.exchange(1, std::memory_order_acquire)) {
            while (f.load(std::memory_order_relaxed)) _mm_pause();
        }
    }
    void unlock() { f.store(0, std::memory_order_release); }
};

}  // namespace

// build::sample_level (src/hnsw/build.rs:19-28).
uint8_t sample_level(uint64_t seed, uint32_t id, double ml) {
    uint64_t h = mix64(seed ^ mix64(uint64_t(id) + 0x9E3779B97F4A7C15ULL));
    double u = double((h >> 11) + 1) * (1.0 / double(1ULL << 53));
    double level = std::floor(-std::log(u) * ml);
    if (level >= double(kMaxLevel)) return kMaxLevel;
    return uint8_t(level);
}

struct Builder::Impl {
    std::unique_ptr<SpinLock[]> locks;
    size_t nlocks = 0;
    std::mutex promotion;
    struct Scratch {
        std::vector<uint16_t> marks;
        uint16_t epoch = 0;
        std::vector<Cand> cand_heap, res_heap;
    };
    std::vector<Scratch> scratch;
};

Builder::Builder(uint32_t dim, int metric, const Params& p) : impl_(new Impl) {
    ix_.dim = dim;
    ix_.metric = metric;
    ix_.params = p;
}
Builder::~Builder() = default;

Err Builder::prepare(const float* v, std::vector<float>* out) const {
    double norm;
    int s = check_vector(v, ix_.dim, &norm);
    if (s) return fail(s);
    if (ix_.metric == HNSW_METRIC_COSINE) {
        if (norm == 0.0) return fail(HNSW_ERR_ZERO_VECTOR);
        double inv = 1.0 / std::sqrt(norm);
        for (uint32_t i = 0; i < ix_.dim; ++i) out->push_back(float(double(v[i]) * inv));
    } else {
        out->insert(out->end(), v, v + ix_.dim);
    }
    return Err();
}

uint32_t Builder::push_nodes(const uint64_t* keys, size_t count) {
    uint32_t first = uint32_t(ix_.node_count());
    size_t total = first + count;
    ix_.l0.resize(total * (ix_.params.m0 + 1), 0);
    ix_.upper.resize(total);
    ix_.levels.resize(total);
    parallel_chunks(count, [&](size_t b, size_t e) {
        for (size_t i = b; i < e; ++i) {
            const uint32_t id = first + uint32_t(i);
            const uint8_t level = sample_level(ix_.params.seed, id, ix_.params.level_multiplier);
            ix_.levels[id] = level;
            if (level) ix_.upper[id].assign(size_t(level) * (ix_.params.m + 1), 0);
        }
    });
    ix_.keys.insert(ix_.keys.end(), keys, keys + count);
    ix_.deleted.resize(total, 0);
    ix_.key_to_id.reserve(ix_.key_to_id.size() + count);
    for (size_t i = 0; i < count; ++i) ix_.key_to_id[keys[i]] = first + uint32_t(i);
    if (impl_->nlocks < total) {
        size_t cap = std::max(total, impl_->nlocks * 2);
        impl_->locks.reset(new SpinLock[cap]);
        impl_->nlocks = cap;
    }
    if (ix_.quantized) {
        // Codes are derived on the device from offsets and scale; nothing to store.
    }
    return first;
}

Err Builder::insert(uint64_t key, const float* v) {
    if (ix_.key_to_id.count(key)) {
        Err e = fail(HNSW_ERR_DUPLICATE_KEY);
        e.a = key;
        return e;
    }
    if (ix_.node_count() >= kMaxNodes) return fail(HNSW_ERR_CAPACITY_EXCEEDED);
    std::vector<float> prepared;
    Err e = prepare(v, &prepared);
    if (e) return e;
    ix_.vectors.insert(ix_.vectors.end(), prepared.begin(), prepared.end());
    uint32_t id = push_nodes(&key, 1);
    if (impl_->scratch.empty()) impl_->scratch.resize(1);
    link(id, 0);
    return Err();
}

Err Builder::insert_batch(const uint64_t* keys, const float* v, size_t count, int threads) {
    uint32_t first = 0;
    Err e = append_batch(keys, v, count, &first);
    if (e) return e;
    link_range(first, threads);
    return Err();
}

Err Builder::append_batch(const uint64_t* keys, const float* v, size_t count, uint32_t* first_out) {
    // prepare_batch: every row is checked in parallel (read only); the error
    // reported is the first failing row's, as in a sequential pass.
    const size_t dim = ix_.dim, base = ix_.vectors.size();
    std::atomic<size_t> first_bad{count};
    int bad_status = 0;
    std::mutex err_mu;
    const bool cosine = ix_.metric == HNSW_METRIC_COSINE;
    parallel_chunks(count, [&](size_t b, size_t e) {
        for (size_t i = b; i < e && i < first_bad.load(std::memory_order_relaxed); ++i) {
            double norm = 0.0;
            int st = check_vector(v + i * dim, dim, &norm);
            if (!st && cosine && norm == 0.0) st = HNSW_ERR_ZERO_VECTOR;
            if (st) {
                std::lock_guard<std::mutex> lock(err_mu);
                if (i < first_bad.load()) {
                    first_bad.store(i);
                    bad_status = st;
                }
                return;
            }
        }
    });
    if (first_bad.load() < count) return fail(bad_status);
    // Duplicate keys: the first key (in batch order) that is live or repeats
    // an earlier one, found with an open-addressing set.
    {
        size_t cap = 16;
        while (cap < 2 * count) cap <<= 1;
        std::vector<uint64_t> table(cap, 0);
        std::vector<uint8_t> used(cap, 0);
        for (size_t i = 0; i < count; ++i) {
            const uint64_t k = keys[i];
            bool dup = ix_.key_to_id.count(k) != 0;
            if (!dup) {
                size_t h = size_t(mix64(k)) & (cap - 1);
                while (used[h] && table[h] != k) h = (h + 1) & (cap - 1);
                if (used[h]) dup = true;
                else {
                    used[h] = 1;
                    table[h] = k;
                }
            }
            if (dup) {
                Err e = fail(HNSW_ERR_DUPLICATE_KEY);
                e.a = k;
                return e;
            }
        }
    }
    if (kMaxNodes - ix_.node_count() < count) return fail(HNSW_ERR_CAPACITY_EXCEEDED);
    ix_.vectors.insert(ix_.vectors.end(), v, v + count * dim);
    if (cosine)
        // vector::normalized (src/vector.rs:42-45), in place.
        parallel_chunks(count, [&](size_t b, size_t e) {
            for (size_t i = b; i < e; ++i) {
                float* row = ix_.vectors.data() + base + i * dim;
                double norm = 0.0;
                check_vector(row, dim, &norm);
                const double inv = 1.0 / std::sqrt(norm);
                for (size_t j = 0; j < dim; ++j) row[j] = float(double(row[j]) * inv);
            }
        });
    *first_out = push_nodes(keys, count);
    return Err();
}

void Builder::truncate(uint32_t first) {
    for (size_t id = first; id < ix_.node_count(); ++id) {
        auto it = ix_.key_to_id.find(ix_.keys[id]);
        if (it != ix_.key_to_id.end() && it->second == id) ix_.key_to_id.erase(it);
    }
    ix_.vectors.resize(size_t(first) * ix_.dim);
    ix_.keys.resize(first);
    ix_.levels.resize(first);
    ix_.deleted.resize(first);
    ix_.l0.resize(size_t(first) * (ix_.params.m0 + 1));
    ix_.upper.resize(first);
}

void Builder::link_range(uint32_t first, int threads) {
    // link_parallel (src/hnsw/mod.rs:340-349)
    uint32_t end = uint32_t(ix_.node_count()), next = first;
    int nt = threads > 0 ? threads : int(std::max(1u, std::thread::hardware_concurrency()));
    if (impl_->scratch.size() < size_t(nt)) impl_->scratch.resize(size_t(nt));
    if (next < end && !ix_.has_entry()) link(next++, 0);
    std::atomic<uint32_t> cursor{next};
    auto worker = [&](int t) {
        for (;;) {
            uint32_t id = cursor.fetch_add(1, std::memory_order_relaxed);
            if (id >= end) break;
            link(id, t);
        }
    };
    if (nt == 1) worker(0);
    else {
        std::vector<std::thread> pool;
        for (int t = 0; t < nt; ++t) pool.emplace_back(worker, t);
        for (auto& th : pool) th.join();
    }
}

std::unique_ptr<Builder> Builder::compacted_unlinked() const {
    const size_t n = ix_.node_count();
    size_t live = 0;
    for (size_t id = 0; id < n; ++id) live += ix_.deleted[id] ? 0 : 1;
    if (live == n) return nullptr;
    std::unique_ptr<Builder> fresh(new Builder(ix_.dim, ix_.metric, ix_.params));
    std::vector<uint64_t> keys;
    keys.reserve(live);
    fresh->ix_.vectors.reserve(live * ix_.dim);
    for (size_t id = 0; id < n; ++id) {
        if (ix_.deleted[id]) continue;
        keys.push_back(ix_.keys[id]);
        const float* row = ix_.vector(uint32_t(id));
        fresh->ix_.vectors.insert(fresh->ix_.vectors.end(), row, row + ix_.dim);
    }
    fresh->push_nodes(keys.data(), keys.size());
    return fresh;
}

void Builder::compact(int threads) {
    std::unique_ptr<Builder> fresh = compacted_unlinked();
    if (!fresh) return;
    fresh->link_range(0, threads);
    if (ix_.quantized) fresh->enable_quantization();
    std::swap(ix_, fresh->ix_);
    std::swap(impl_, fresh->impl_);
}

bool Builder::remove(uint64_t key) {
    auto it = ix_.key_to_id.find(key);
    if (it == ix_.key_to_id.end()) return false;
    ix_.deleted[it->second] = 1;
    ix_.key_to_id.erase(it);
    return true;
}

// ScalarQuantizer::train (src/quantization.rs:32-56).
void Builder::enable_quantization() {
    size_t dim = ix_.dim, rows = ix_.node_count();
    std::vector<float> offset(dim, 0.0f);
    if (ix_.metric == HNSW_METRIC_L2 && rows > 0) {
        std::vector<double> sum(dim, 0.0);
        for (size_t r = 0; r < rows; ++r)
            for (size_t j = 0; j < dim; ++j) sum[j] += double(ix_.vectors[r * dim + j]);
        for (size_t j = 0; j < dim; ++j) offset[j] = float(sum[j] / double(rows));
    }
    float max_abs = 0.0f;
    for (size_t r = 0; r < rows; ++r)
        for (size_t j = 0; j < dim; ++j) max_abs = std::max(max_abs, std::fabs(ix_.vectors[r * dim + j] - offset[j]));
    ix_.q_offset = offset;
    ix_.q_scale = (max_abs > 0.0f && std::isfinite(max_abs)) ? max_abs / 127.0f : 1.0f;
    ix_.quantized = true;
}

// HnswIndex::link (src/hnsw/build.rs:41-94) and its helpers.
void Builder::link(uint32_t id, int thread) {
    HostIndex& ix = ix_;
    Impl& im = *impl_;
    const Params& P = ix.params;
    const uint32_t dim = ix.dim;
    const int metric = ix.metric;
    const float* query = ix.vector(id);
    auto dist = [&](uint32_t other) { return metric_distance(metric, query, ix.vector(other), dim); };
    auto read_list = [&](uint32_t node, unsigned layer, std::vector<uint32_t>& out) {
        out.clear();
        const uint32_t* blk = ix.block(node, layer);
        uint32_t cnt = std::min(__atomic_load_n(blk, __ATOMIC_ACQUIRE), ix.capacity(layer));
        for (uint32_t j = 0; j < cnt; ++j) out.push_back(__atomic_load_n(blk + 1 + j, __ATOMIC_RELAXED));
    };
    auto set_list = [&](uint32_t node, unsigned layer, const uint32_t* ids, size_t cnt) {
        uint32_t* blk = ix.block(node, layer);
        for (size_t j = 0; j < cnt; ++j) __atomic_store_n(blk + 1 + j, ids[j], __ATOMIC_RELAXED);
        __atomic_store_n(blk, uint32_t(cnt), __ATOMIC_RELEASE);
    };
    auto try_push = [&](uint32_t node, unsigned layer, uint32_t nb) {
        uint32_t* blk = ix.block(node, layer);
        uint32_t c = __atomic_load_n(blk, __ATOMIC_RELAXED);
        if (c >= ix.capacity(layer)) return false;
        __atomic_store_n(blk + 1 + c, nb, __ATOMIC_RELAXED);
        __atomic_store_n(blk, c + 1, __ATOMIC_RELEASE);
        return true;
    };
    std::vector<uint32_t> tmp;

    auto greedy = [&](Cand best, unsigned layer) {
        std::vector<uint32_t> nb;
        for (;;) {
            uint32_t from = best.id;
            read_list(from, layer, nb);
            for (uint32_t n : nb) {
                float d = dist(n);
                if (d < best.d) best = Cand{d, n};
            }
            if (best.id == from) return best;
        }
    };

    Impl::Scratch& sc = im.scratch[size_t(thread)];
    auto search_layer = [&](const std::vector<Cand>& eps, size_t ef, unsigned layer) {
        size_t n = ix.node_count();
        if (sc.marks.size() < n) sc.marks.resize(n, 0);
        sc.epoch = uint16_t(sc.epoch + 1);
        if (sc.epoch == 0) {
            std::fill(sc.marks.begin(), sc.marks.end(), 0);
            sc.epoch = 1;
        }
        auto visit = [&](uint32_t v) {
            if (sc.marks[v] == sc.epoch) return false;
            sc.marks[v] = sc.epoch;
            return true;
        };
        auto& C = sc.cand_heap;
        auto& R = sc.res_heap;
        C.clear();
        R.clear();
        for (const Cand& ep : eps) {
            if (!visit(ep.id)) continue;
            C.push_back(ep);
            std::push_heap(C.begin(), C.end(), Greater());
            if (ep.id != id) {
                R.push_back(ep);
                std::push_heap(R.begin(), R.end(), Less());
                if (R.size() > ef) {
                    std::pop_heap(R.begin(), R.end(), Less());
                    R.pop_back();
                }
            }
        }
        std::vector<uint32_t> nb;
        while (!C.empty()) {
            std::pop_heap(C.begin(), C.end(), Greater());
            Cand cur = C.back();
            C.pop_back();
            if (R.size() >= ef && !R.empty() && cur.d > R.front().d) break;
            read_list(cur.id, layer, nb);
            for (uint32_t v : nb) {
                if (!visit(v)) continue;
                float d = dist(v);
                bool improves = R.size() < ef || (!R.empty() && d < R.front().d);
                if (!improves) continue;
                Cand c{d, v};
                C.push_back(c);
                std::push_heap(C.begin(), C.end(), Greater());
                if (v != id) {
                    R.push_back(c);
                    std::push_heap(R.begin(), R.end(), Less());
                    if (R.size() > ef) {
                        std::pop_heap(R.begin(), R.end(), Less());
                        R.pop_back();
                    }
                }
            }
        }
        std::vector<Cand> out(R.begin(), R.end());
        std::sort(out.begin(), out.end(), Less());
        return out;
    };

    // select_neighbors (build.rs:152-198), extend_candidates (build.rs:202-222)
    auto select = [&](uint32_t base_id, const float* base, const std::vector<Cand>& cands, size_t m,
                      unsigned layer) {
        std::vector<uint32_t> out;
        if (P.selection == 0) {
            for (size_t i = 0; i < cands.size() && i < m; ++i) out.push_back(cands[i].id);
            return out;
        }
        std::vector<Cand> extended;
        const std::vector<Cand>* pool = &cands;
        if (P.extend_candidates) {
            std::unordered_set<uint32_t> seen;
            for (const Cand& c : cands) seen.insert(c.id);
            seen.insert(base_id);
            extended = cands;
            std::vector<uint32_t> nb;
            for (const Cand& c : cands) {
                read_list(c.id, layer, nb);
                for (uint32_t v : nb)
                    if (seen.insert(v).second)
                        extended.push_back(Cand{metric_distance(metric, base, ix.vector(v), dim), v});
            }
            std::sort(extended.begin(), extended.end(), Less());
            pool = &extended;
        }
        std::vector<Cand> selected, discarded;
        for (const Cand& c : *pool) {
            if (selected.size() >= m) break;
            const float* v = ix.vector(c.id);
            bool diverse = true;
            for (const Cand& s : selected)
                if (!(metric_distance(metric, v, ix.vector(s.id), dim) >= c.d)) {
                    diverse = false;
                    break;
                }
            if (diverse) selected.push_back(c);
            else if (P.keep_pruned) discarded.push_back(c);
        }
        size_t room = m - selected.size();
        for (size_t i = 0; i < discarded.size() && i < room; ++i) selected.push_back(discarded[i]);
        for (const Cand& c : selected) out.push_back(c.id);
        return out;
    };

    auto write_shrunk = [&](uint32_t node, const std::vector<uint32_t>& ids, unsigned layer) {
        size_t cap = ix.capacity(layer);
        if (ids.size() <= cap) {
            set_list(node, layer, ids.data(), ids.size());
            return;
        }
        const float* base = ix.vector(node);
        std::vector<Cand> cands;
        cands.reserve(ids.size());
        for (uint32_t c : ids) cands.push_back(Cand{metric_distance(metric, base, ix.vector(c), dim), c});
        std::sort(cands.begin(), cands.end(), Less());
        std::vector<uint32_t> sel = select(node, base, cands, cap, layer);
        set_list(node, layer, sel.data(), sel.size());
    };

    auto install_own = [&](const std::vector<uint32_t>& selected, unsigned layer) {
        im.locks[id].lock();
        std::vector<uint32_t> merged;
        read_list(id, layer, merged);
        if (merged.empty()) set_list(id, layer, selected.data(), selected.size());
        else {
            for (uint32_t v : selected)
                if (std::find(merged.begin(), merged.end(), v) == merged.end()) merged.push_back(v);
            write_shrunk(id, merged, layer);
        }
        im.locks[id].unlock();
    };

    auto connect = [&](uint32_t node, uint32_t nw, unsigned layer) {
        im.locks[node].lock();
        std::vector<uint32_t> current;
        read_list(node, layer, current);
        if (std::find(current.begin(), current.end(), nw) == current.end() && !try_push(node, layer, nw)) {
            current.push_back(nw);
            write_shrunk(node, current, layer);
        }
        im.locks[node].unlock();
    };

    const unsigned level = ix.levels[id];
    uint64_t entry = __atomic_load_n(&ix.entry_word, __ATOMIC_ACQUIRE);
    std::unique_lock<std::mutex> promotion;
    if (entry == ~0ull || level > uint32_t(entry >> 32)) {
        std::unique_lock<std::mutex> guard(im.promotion);
        entry = __atomic_load_n(&ix.entry_word, __ATOMIC_ACQUIRE);
        if (entry == ~0ull) {
            __atomic_store_n(&ix.entry_word, (uint64_t(level) << 32) | id, __ATOMIC_RELEASE);
            return;
        }
        if (level > uint32_t(entry >> 32)) promotion = std::move(guard);
    }
    uint32_t entry_id = uint32_t(entry), top = uint32_t(entry >> 32);
    Cand ep{dist(entry_id), entry_id};
    for (unsigned layer = top; layer > level; --layer) ep = greedy(ep, layer);
    size_t ef = std::max<size_t>(P.ef_construction, P.m);
    std::vector<Cand> eps{ep};
    for (int layer = int(std::min(level, top)); layer >= 0; --layer) {
        std::vector<Cand> found = search_layer(eps, ef, unsigned(layer));
        std::vector<uint32_t> selected = select(id, query, found, P.m, unsigned(layer));
        install_own(selected, unsigned(layer));
        for (uint32_t nbr : selected) connect(nbr, id, unsigned(layer));
        if (!found.empty()) eps = std::move(found);
    }
    if (promotion.owns_lock()) __atomic_store_n(&ix.entry_word, (uint64_t(level) << 32) | id, __ATOMIC_RELEASE);
    (void)tmp;
}

}  // namespace hnswgpu
